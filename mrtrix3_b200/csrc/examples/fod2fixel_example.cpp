// fod2fixel's segmentation through the C ABI: the segmenter on the built-in
// 1281-direction set (csd_fmls_create_default, as Segmenter (dirs, lmax)
// with load_fmls_thresholds' defaults), then one csd_fmls_segment over a
// batch of FODs on the device.
// Build (one command line):
//   g++ -std=c++17 -O2 -I include -I /usr/local/cuda/include
//       mrtrix3_b200/csrc/examples/fod2fixel_example.cpp -L mrtrix3_b200 -lcsd_b200
//       -L /usr/local/cuda/lib64 -lcudart -Wl,-rpath,$PWD/mrtrix3_b200 -o fod2fixel_example
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "csd_b200.h"

int main() {
  const int lmax = 8, nsh = 45, n = 2, room = 16;
  csd_fmls* fmls = nullptr;
  if (csd_fmls_create_default(lmax, 0.0, 0.1, 1.0, &fmls)) {
    std::fprintf(stderr, "%s\n", csd_last_error());
    return 1;
  }
  // voxel 0: an FOD symmetric about z (l = 0 and l = 2, m = 0 terms: one lobe
  // along z); voxel 1: its DC term negative (no lobes)
  std::vector<float> fod(n * nsh, 0.0f);
  fod[0] = 0.5f;
  fod[3] = 0.4f;  // index l (l + 1) / 2 + m of l = 2, m = 0
  fod[nsh] = -0.5f;
  float *d_fod = nullptr, *d_fixels = nullptr;
  int32_t* d_counts = nullptr;
  if (cudaMalloc(&d_fod, fod.size() * sizeof(float)) || cudaMalloc(&d_counts, n * sizeof(int32_t)) ||
      cudaMalloc(&d_fixels, (size_t)n * room * 8 * sizeof(float)))
    return 1;
  cudaMemcpy(d_fod, fod.data(), fod.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (csd_fmls_segment(fmls, d_fod, n, nsh, 1, nullptr, room, d_counts, d_fixels, nullptr)) {
    std::fprintf(stderr, "%s\n", csd_last_error());
    return 1;
  }
  std::vector<int32_t> counts(n);
  std::vector<float> fixels((size_t)n * room * 8);
  cudaMemcpy(counts.data(), d_counts, counts.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
  cudaMemcpy(fixels.data(), d_fixels, fixels.size() * sizeof(float), cudaMemcpyDeviceToHost);
  for (int v = 0; v < n; ++v) {
    std::printf("voxel %d: %d fixel(s)\n", v, counts[v]);
    for (int q = 0; q < counts[v] && q < room; ++q) {
      const float* f = &fixels[((size_t)v * room + q) * 8];
      std::printf("  dir [%.4f %.4f %.4f]  afd %.4f  peak %.4f\n", f[0], f[1], f[2], f[6], f[7]);
    }
  }
  cudaFree(d_fod);
  cudaFree(d_counts);
  cudaFree(d_fixels);
  csd_fmls_destroy(fmls);
  return 0;
}
