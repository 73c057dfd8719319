// C++ drop-in for MRtrix3's MR::DWI::SDeconv::CSD (src/dwi/sdeconv/csd.h:
// 46-281) over the libcsd_b200 C ABI.  Code written against the reference's
// surface -- Shared(header) / parse_cmdline_options() / set_response() /
// init() / nSH(), and a CSD(shared) object with set() / iterate() / FOD() --
// keeps compiling; the per-voxel object runs each call as a batch of one on
// the GPU (correct, not fast), and dwi2fod_csd() is the batched replacement
// of the ThreadedLoop over CSD_Processor (cmd/dwi2fod.cpp:120-176, 275-281).
//
// Differences from the reference, by design: no Eigen (std::vector<double>
// stands in for Eigen vectors/matrices, row-major), the header is replaced
// by the gradient table, and options arrive as a struct instead of App.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "csd_b200.h"

namespace MR {
namespace DWI {
namespace SDeconv {

// The option group of csd.cpp:318-346 (+ -lmax / -directions, dwi2fod.cpp:38-59).
struct CSDOptions {
  std::vector<uint32_t> lmax;          // -lmax (a single value)
  std::vector<double> filter;          // -filter
  std::vector<double> directions;      // -directions, [n][2] az/el row-major
  double neg_lambda = 1.0;             // -neg_lambda
  double norm_lambda = 1.0;            // -norm_lambda
  double threshold = 0.0;              // -threshold
  size_t niter = 50;                   // -niter
  std::vector<double> shells;          // -shells (one non-b=0 shell; the constructor's
                                       // select_shells at csd.h:64 -- applied by init())
  bool has_neg_lambda = false, has_norm_lambda = false, has_threshold = false, has_niter = false;
};

class Exception : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

inline void check(int rc) {
  if (rc != CSD_OK) throw Exception(csd_last_error());
}

class CSD {
 public:
  class Shared {
   public:
    // csd.h:52-68: the gradient table [n_volumes][4] (x y z b) stands in for the header
    explicit Shared(const std::vector<double>& grad_table) : grad(grad_table) {
      if (grad.empty() || grad.size() % 4) throw Exception("gradient table must be [n][4]");
    }
    Shared(const Shared&) = delete;
    Shared& operator=(const Shared&) = delete;
    ~Shared() { csd_shared_destroy(handle_); }

    // csd.h:71-99
    void parse_cmdline_options(const CSDOptions& opt) {
      if (!opt.lmax.empty()) {
        if (opt.lmax.size() != 1) throw Exception("CSD algorithm expects a single lmax to be specified");
        lmax_cmdline = opt.lmax.front();
      }
      if (!opt.filter.empty()) init_filter = opt.filter;
      if (!opt.directions.empty()) HR_dirs = opt.directions;
      if (opt.has_neg_lambda) neg_lambda = opt.neg_lambda;
      if (opt.has_norm_lambda) norm_lambda = opt.norm_lambda;
      if (opt.has_threshold) threshold = opt.threshold;
      if (opt.has_niter) niter = opt.niter;
      if (!opt.shells.empty()) shells = opt.shells;
    }

    // csd.h:102-114
    void set_response(const std::string& path) {
      std::ifstream f(path);
      if (!f) throw Exception("cannot open response file \"" + path + "\"");
      std::vector<double> v;
      std::string line;
      while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ss(line);
        double x;
        while (ss >> x) v.push_back(x);
      }
      set_response(v);
    }
    template <class VectorType>
    void set_response(const VectorType& in) {
      response.assign(in.begin(), in.end());
      lmax_response = response.empty() ? 0 : 2 * (uint32_t(response.size()) - 1);
    }

    // csd.h:117-198 (host FP64 precompute inside the library)
    void init() {
      csd_params p;
      csd_params_init(&p);
      p.lmax = int(lmax_cmdline);
      p.niter = int(niter);
      p.neg_lambda = neg_lambda;
      p.norm_lambda = norm_lambda;
      p.threshold = threshold;
      p.filter = init_filter.empty() ? nullptr : init_filter.data();
      p.n_filter = int(init_filter.size());
      p.shells = shells.empty() ? nullptr : shells.data();
      p.n_shells = int(shells.size());
      csd_shared* h = nullptr;
      check(csd_shared_create(&p, grad.data(), int(grad.size() / 4), response.data(), int(response.size()),
                              HR_dirs.empty() ? nullptr : HR_dirs.data(), int(HR_dirs.size() / 2), &h));
      csd_shared_destroy(handle_);
      handle_ = h;
      int info[8];
      check(csd_shared_info(h, info));
      lmax = info[0];
      lmax_response = info[1];
      lmax_data = info[2];
      nsh_ = size_t(info[3]);
      std::vector<int> d(static_cast<size_t>(info[5]));
      check(csd_shared_dwis(h, d.data()));
      dwis.assign(d.begin(), d.end());
    }

    size_t nSH() const { return nsh_; }  // csd.h:200-202
    csd_shared* handle() const { return handle_; }

    // the public members of csd.h:204-211 that callers read
    std::vector<double> grad, response, init_filter, HR_dirs, shells;
    double neg_lambda = 1.0, norm_lambda = 1.0, threshold = 0.0;
    std::vector<size_t> dwis;
    uint32_t lmax_response = 0, lmax_data = 0, lmax_cmdline = 0, lmax = 0;
    size_t niter = 50;

   private:
    csd_shared* handle_ = nullptr;
    size_t nsh_ = 0;
  };

  // csd.h:221-230 (holds a reference: `shared` must outlive the object)
  explicit CSD(const Shared& shared_data) : shared(shared_data) {
    check(csd_state_create(shared.handle(), 1, &state_));
    const size_t nvol = shared.grad.size() / 4;
    const size_t words = (nvol > shared.nSH() ? nvol : shared.nSH()) + 16;  // record, or FOD + status
    if (cudaMalloc(&d_rec_, words * sizeof(float)) != cudaSuccess) throw Exception("cudaMalloc failed");
    F_.assign(shared.nSH(), 0.0);
  }
  CSD(const CSD& o) : CSD(o.shared) {}
  ~CSD() {
    csd_state_destroy(state_);
    cudaFree(d_rec_);
  }

  // csd.h:237-243: DW_signals are the samples of the selected shell (dwis order).
  // Unlike the reference's set(), which takes the samples as given, this one
  // goes through csd_state_set and so also applies dwi2fod's load_data rules
  // (cmd/dwi2fod.cpp:156-173): negative samples are clamped to zero, and a
  // non-finite sample leaves F at zero with iterate() never returning true.
  // dwi2fod applies the same rules before calling set(), so its results are
  // unchanged; a caller that hands set() negative samples directly gets the
  // fit of the clamped samples.
  template <class VectorType>
  void set(const VectorType& DW_signals) {
    const size_t nvol = shared.grad.size() / 4;
    std::vector<float> rec(nvol, 0.f);
    size_t i = 0;
    for (auto v : DW_signals) {
      if (i >= shared.dwis.size()) break;
      rec[shared.dwis[i++]] = float(v);
    }
    if (cudaMemcpy(d_rec_, rec.data(), nvol * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      throw Exception("cudaMemcpy failed");
    check(csd_state_set(state_, d_rec_, 1, int64_t(nvol), 1, nullptr, nullptr));
    done_ = false;
  }

  // csd.h:245-269: true once the negative set repeats
  bool iterate() {
    if (done_) return true;
    int64_t active = 0;
    check(csd_state_iterate(state_, &active, nullptr));
    uint8_t st = 0;
    fetch(&st);
    done_ = (st & 0x0F) == CSD_STATUS_CONVERGED;
    return done_;
  }

  // csd.h:271
  const std::vector<double>& FOD() const {
    const_cast<CSD*>(this)->fetch(nullptr);
    return F_;
  }

  const Shared& shared;

 private:
  void fetch(uint8_t* status) {
    const size_t n = shared.nSH();
    float* d_out = d_rec_;  // the record is no longer needed once set() has run
    uint8_t* d_st = reinterpret_cast<uint8_t*>(d_out + n);
    check(csd_state_fod(state_, d_out, int64_t(n), d_st, nullptr, nullptr, nullptr));
    std::vector<float> f(n);
    if (cudaMemcpy(f.data(), d_out, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess ||
        (status && cudaMemcpy(status, d_st, 1, cudaMemcpyDeviceToHost) != cudaSuccess))
      throw Exception("cudaMemcpy failed");
    F_.assign(f.begin(), f.end());
  }

  csd_state* state_ = nullptr;
  float* d_rec_ = nullptr;
  std::vector<double> F_;
  bool done_ = false;
};

// dwi2fod csd over a whole volume on host buffers: dwi [n][n_volumes]
// voxel-interleaved float32, optional mask, fod [n][nSH] (cmd/dwi2fod.cpp:275-281).
inline void dwi2fod_csd(const CSD::Shared& shared, const float* dwi, int64_t n_voxels, const uint8_t* mask,
                        float* fod, uint8_t* status = nullptr, uint8_t* iterations = nullptr) {
  check(csd_dwi2fod_host(shared.handle(), dwi, n_voxels, mask, fod, status, iterations));
}

}  // namespace SDeconv
}  // namespace DWI
}  // namespace MR
