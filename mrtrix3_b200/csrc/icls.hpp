// C++ drop-in for MRtrix3's Math::ICLS::Problem / Solver
// (core/math/constrained_least_squares.h:71-370) over the libcsd_b200 C ABI,
// as dwi2fod msmt_csd (MSMT_CSD::Shared::init, src/dwi/sdeconv/msmt_csd.h:
// 203-204) and amp2response (cmd/amp2response.cpp:345-346) build and use
// them.  The problem's tables live on the GPU; Solver::operator() solves one
// right-hand side as the reference does (FP64, synchronous), solve_batch()
// many on host buffers at once (csd_icls_solve_host).
//
// Differences from the reference, by design: no Eigen (std::vector<double>,
// row-major, stands in for Eigen matrices and vectors); the second
// constructor's separate equality matrix is passed stacked under the
// inequalities with its row count, as the first constructor takes it.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "csd_b200.h"

namespace MR {
namespace Math {
namespace ICLS {

class Exception : public std::runtime_error {
 public:
  using std::runtime_error::runtime_error;
};

inline void icls_check(int rc) {
  if (rc != CSD_OK) throw Exception(csd_last_error());
}

template <typename ValueType = double>
class Problem {
 public:
  // min ||H x - b||^2 s.t. A x >= t (the last num_equalities rows of A as
  // equalities); H [rows][cols] (or H^T H [cols][cols] when
  // problem_in_standard_form), A [ncons][cols], t empty or [ncons]
  Problem(const std::vector<double>& problem_matrix, size_t rows, size_t cols,
          const std::vector<double>& inequality_constraint_matrix, size_t ncons,
          const std::vector<double>& inequality_constraint_vector = {}, size_t num_equalities = 0,
          double solution_min_norm_regularisation = 0.0, double constraint_min_norm_regularisation = 0.0,
          size_t max_iterations = 0, double tolerance = 0.0, bool problem_in_standard_form = false)
      : rows_(problem_in_standard_form ? cols : rows), cols_(cols), ncons_(ncons), num_eq_(num_equalities) {
    if (problem_matrix.size() != rows * cols || inequality_constraint_matrix.size() != ncons * cols)
      throw Exception("FIXME: dimensions of problem and constraint matrices do not match (ICLS)");
    if (!inequality_constraint_vector.empty() && inequality_constraint_vector.size() != ncons)
      throw Exception("FIXME: dimensions of constraint matrix and vector do not match (ICLS)");
    const double* t = inequality_constraint_vector.empty() ? nullptr : inequality_constraint_vector.data();
    if (problem_in_standard_form)
      icls_check(csd_icls_create_standard(problem_matrix.data(), (int)cols, inequality_constraint_matrix.data(),
                                          (int)ncons, t, (int)num_equalities, solution_min_norm_regularisation,
                                          constraint_min_norm_regularisation, (int)max_iterations, tolerance, &h_));
    else
      icls_check(csd_icls_create(problem_matrix.data(), (int)rows, (int)cols, inequality_constraint_matrix.data(),
                                 (int)ncons, t, (int)num_equalities, solution_min_norm_regularisation,
                                 constraint_min_norm_regularisation, (int)max_iterations, tolerance, &h_));
  }
  Problem(const Problem&) = delete;
  Problem& operator=(const Problem&) = delete;
  Problem(Problem&& o) noexcept : h_(std::exchange(o.h_, nullptr)), rows_(o.rows_), cols_(o.cols_),
                                  ncons_(o.ncons_), num_eq_(o.num_eq_) {}
  ~Problem() { csd_icls_destroy(h_); }

  size_t num_parameters() const { return cols_; }
  size_t num_measurements() const { return rows_; }
  size_t num_constraints() const { return ncons_; }
  size_t num_equalities() const { return num_eq_; }
  csd_icls* handle() const { return h_; }

 private:
  csd_icls* h_ = nullptr;
  size_t rows_, cols_, ncons_, num_eq_;
};

template <typename ValueType = double>
class Solver {
 public:
  explicit Solver(const Problem<ValueType>& problem) : P(problem) {}

  // x for one right-hand side b (b: the measurements, or H^T b for a problem
  // in standard form); returns the solver's rounds, as the reference does
  size_t operator()(std::vector<double>& x, const std::vector<double>& b) {
    if (b.size() != P.num_measurements()) throw Exception("ICLS: right-hand side of the wrong size");
    x.assign(P.num_parameters(), 0.0);
    double *db = nullptr, *dx = nullptr;
    int32_t *dn = nullptr, niter = 0;
    cudaError_t e = cudaMalloc(&db, b.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dx, x.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&dn, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpy(db, b.data(), b.size() * sizeof(double), cudaMemcpyHostToDevice);
    int rc = CSD_OK;
    if (e == cudaSuccess)
      rc = csd_icls_solve_f64(P.handle(), db, 1, (int64_t)b.size(), 1, dx, (int64_t)x.size(), dn, nullptr);
    if (e == cudaSuccess && rc == CSD_OK) e = cudaMemcpy(x.data(), dx, x.size() * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && rc == CSD_OK) e = cudaMemcpy(&niter, dn, sizeof(int32_t), cudaMemcpyDeviceToHost);
    cudaFree(db);
    cudaFree(dx);
    cudaFree(dn);
    icls_check(rc);
    if (e != cudaSuccess) throw Exception(std::string("ICLS: ") + cudaGetErrorString(e));
    return (size_t)niter;
  }

  // many right-hand sides on host buffers: b [n][num_measurements] float,
  // x [n][num_parameters], niter [n] or nullptr (csd_icls_solve_host)
  void solve_batch(const float* b, int64_t n, float* x, int32_t* niter = nullptr, const uint8_t* mask = nullptr) {
    icls_check(csd_icls_solve_host(P.handle(), b, n, (int64_t)P.num_measurements(), mask, x, niter, nullptr));
  }

  const Problem<ValueType>& problem() const { return P; }

 private:
  const Problem<ValueType>& P;
};

}  // namespace ICLS
}  // namespace Math
}  // namespace MR
