// fod2fixel's per-voxel loop written against the FMLS drop-in (fmls.hpp):
// the Segmenter with load_fmls_thresholds' -fmls_no_thresholds, one voxel
// through operator() as the reference's worker threads call it, then a
// whole batch of voxels through segment().
// Build (one command line):
//   g++ -std=c++17 -O2 -I include -I mrtrix3_b200/csrc -I /usr/local/cuda/include
//       mrtrix3_b200/csrc/examples/fmls_segmenter_example.cpp -L mrtrix3_b200 -lcsd_b200
//       -L /usr/local/cuda/lib64 -lcudart -Wl,-rpath,$PWD/mrtrix3_b200 -o fmls_segmenter_example
#include <cstdio>
#include <vector>

#include "fmls.hpp"

int main() {
  using namespace MR::DWI::FMLS;
  Segmenter fmls(8);
  fmls.set_integral_threshold(0.0);   // -fmls_no_thresholds
  fmls.set_peak_value_threshold(0.0);
  SH_coefs in(45, 0.0);
  in[0] = 0.5;
  in[3] = 0.4;  // l = 2, m = 0: one lobe along z
  FOD_lobes lobes;
  fmls(in, lobes);
  for (const auto& lobe : lobes)
    std::printf("lobe: dir [%.4f %.4f %.4f] integral %.4f peak %.4f\n", lobe.get_mean_dir()[0],
                lobe.get_mean_dir()[1], lobe.get_mean_dir()[2], lobe.get_integral(), lobe.get_max_peak_value());
  std::vector<float> rows(3 * 45, 0.0f);
  for (int v = 0; v < 3; ++v) {
    rows[v * 45] = 0.5f;
    rows[v * 45 + 3 + v] = 0.3f;  // l = 2, m = 0 / 1 / 2
  }
  std::vector<FOD_lobes> all;
  fmls.segment(rows.data(), 3, all);
  for (size_t v = 0; v < all.size(); ++v) std::printf("voxel %zu: %zu lobes\n", v, all[v].size());
  return 0;
}
