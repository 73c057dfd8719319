// C++ drop-in for MRtrix3's FMLS FOD segmenter (src/dwi/fmls.h:60-291) over
// the libcsd_b200 C ABI, as fod2fixel (cmd/fod2fixel.cpp:288-330) uses it:
// Segmenter (directions, lmax), the threshold setters of
// load_fmls_thresholds, and operator() (SH_coefs, FOD_lobes&) for one voxel;
// segment() does many voxels of host rows in one launch.  The direction set
// is the built-in 1281-direction tessellation (csd_fmls_create_default);
// the segmentation runs on the GPU in FP64.
//
// Differences from the reference, by design: no Eigen (std::array /
// std::vector stand in); a lobe carries what fod2fixel writes -- its unit
// mean direction, the direction and amplitude of its largest peak, its
// integral -- not its direction mask or per-direction values; the lookup
// table and null lobe (create_lookup_table, create_null_lobe) are not
// produced.  Changing a threshold rebuilds the device tables at the next
// call.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <vector>

#include "csd_b200.h"

namespace MR {
namespace DWI {
namespace FMLS {

class Exception : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

inline void fmls_check(int rc) {
  if (rc != CSD_OK) throw Exception(csd_last_error());
}

// fmls.h:30-32
constexpr double FMLS_INTEGRAL_THRESHOLD_DEFAULT = 0.0;
constexpr double FMLS_PEAK_VALUE_THRESHOLD_DEFAULT = 0.1;
constexpr double FMLS_MERGE_RATIO_BRIDGE_TO_PEAK_DEFAULT = 1.0;

class FOD_lobe {
 public:
  FOD_lobe(const float* f)
      : mean_dir_{f[0], f[1], f[2]}, peak_dir_{f[3], f[4], f[5]}, integral_(f[6]), max_peak_value_(f[7]) {}
  const std::array<double, 3>& get_mean_dir() const { return mean_dir_; }
  const std::array<double, 3>& get_peak_dir(size_t i) const {
    if (i) throw Exception("only the largest peak of a lobe is available");
    return peak_dir_;
  }
  double get_integral() const { return integral_; }
  double get_max_peak_value() const { return max_peak_value_; }
  bool is_negative() const { return false; }  // negative lobes are never kept

 private:
  std::array<double, 3> mean_dir_, peak_dir_;
  double integral_, max_peak_value_;
};

class FOD_lobes : public std::vector<FOD_lobe> {
 public:
  std::array<int, 3> vox{{-1, -1, -1}};
};

class SH_coefs : public std::vector<double> {
 public:
  using std::vector<double>::vector;
  std::array<int, 3> vox{{-1, -1, -1}};
};

class Segmenter {
 public:
  explicit Segmenter(size_t lmax) : lmax_(lmax), nsh_((lmax + 1) * (lmax + 2) / 2) {}
  ~Segmenter() { release(); }
  Segmenter(const Segmenter&) = delete;
  Segmenter& operator=(const Segmenter&) = delete;

  double get_integral_threshold() const { return integral_; }
  void set_integral_threshold(double i) { integral_ = i; dirty_ = true; }
  double get_peak_value_threshold() const { return peak_; }
  void set_peak_value_threshold(double i) { peak_ = i; dirty_ = true; }
  double get_lobe_merge_ratio() const { return merge_; }
  void set_lobe_merge_ratio(double i) { merge_ = i; dirty_ = true; }

  // Segmenter::operator() (fmls.cpp:159-311) for one voxel
  bool operator()(const SH_coefs& in, FOD_lobes& out) {
    if (in.size() != nsh_) throw Exception("SH coefficients do not match the segmenter's lmax");
    std::vector<float> row(in.begin(), in.end());
    std::vector<FOD_lobes> all;
    segment(row.data(), 1, all);
    out = all[0];
    out.vox = in.vox;
    return true;
  }

  // n voxels of host rows [n][nsh] (float, as fod2fixel reads the image):
  // the lobes of each, in the reference's order
  void segment(const float* rows, size_t n, std::vector<FOD_lobes>& out) {
    out.assign(n, FOD_lobes());
    if (!n) return;
    ensure();
    size_t room = 16;
    std::vector<int32_t> counts(n);
    std::vector<float> fixels;
    for (int pass = 0; pass < 2; ++pass) {
      reserve(n, room);
      cuda(cudaMemcpy(d_rows_, rows, n * nsh_ * sizeof(float), cudaMemcpyHostToDevice));
      fmls_check(csd_fmls_segment(h_, d_rows_, (int64_t)n, (int64_t)nsh_, 1, nullptr, (int)room, d_counts_, d_fixels_,
                                  nullptr));
      cuda(cudaMemcpy(counts.data(), d_counts_, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
      size_t most = 0;
      for (int32_t c : counts) most = c > (int32_t)most ? (size_t)c : most;
      if (most <= room) break;
      room = most;  // again with room for every lobe
    }
    fixels.resize(n * room * 8);
    cuda(cudaMemcpy(fixels.data(), d_fixels_, fixels.size() * sizeof(float), cudaMemcpyDeviceToHost));
    for (size_t v = 0; v < n; ++v)
      for (int q = 0; q < counts[v]; ++q) out[v].emplace_back(&fixels[(v * room + q) * 8]);
  }

 private:
  static void cuda(cudaError_t e) {
    if (e != cudaSuccess) throw Exception(cudaGetErrorString(e));
  }
  void ensure() {
    if (h_ && !dirty_) return;
    if (h_) csd_fmls_destroy(h_);
    h_ = nullptr;
    fmls_check(csd_fmls_create_default((int)lmax_, integral_, peak_, merge_, &h_));
    dirty_ = false;
  }
  void reserve(size_t n, size_t room) {
    if (n <= cap_n_ && room <= cap_room_) return;
    free_buffers();
    cuda(cudaMalloc(&d_rows_, n * nsh_ * sizeof(float)));
    cuda(cudaMalloc(&d_counts_, n * sizeof(int32_t)));
    cuda(cudaMalloc(&d_fixels_, n * room * 8 * sizeof(float)));
    cap_n_ = n;
    cap_room_ = room;
  }
  void free_buffers() {
    cudaFree(d_rows_);
    cudaFree(d_counts_);
    cudaFree(d_fixels_);
    d_rows_ = nullptr;
    d_counts_ = nullptr;
    d_fixels_ = nullptr;
    cap_n_ = cap_room_ = 0;
  }
  void release() {
    free_buffers();
    if (h_) csd_fmls_destroy(h_);
    h_ = nullptr;
  }

  size_t lmax_, nsh_;
  double integral_ = FMLS_INTEGRAL_THRESHOLD_DEFAULT, peak_ = FMLS_PEAK_VALUE_THRESHOLD_DEFAULT,
         merge_ = FMLS_MERGE_RATIO_BRIDGE_TO_PEAK_DEFAULT;
  bool dirty_ = true;
  csd_fmls* h_ = nullptr;
  float* d_rows_ = nullptr;
  int32_t* d_counts_ = nullptr;
  float* d_fixels_ = nullptr;
  size_t cap_n_ = 0, cap_room_ = 0;
};

}  // namespace FMLS
}  // namespace DWI
}  // namespace MR
