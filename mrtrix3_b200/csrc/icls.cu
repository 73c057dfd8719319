// Inequality-constrained least squares on the GPU, batched over voxels: the
// solver of MRtrix3's multi-shell multi-tissue CSD (src/dwi/sdeconv/
// msmt_csd.h:249-270) and of core/math/constrained_least_squares.h.
//
// Problem set-up (constrained_least_squares.h:90-151) in FP64 on the host:
// L = chol(H^T H + solution_reg * max diag), b2d = H L^-T, B = A L^-T with
// each row (and its t entry) divided by the row's norm; plus the constraints'
// Gram matrix G = B B^T, from which the active-set systems are read.
//
// Solver (constrained_least_squares.h:241-370), a warp per voxel in FP64:
// y_u = b2d^T b, c_u = B y_u - t; while the most violated inequality has
// c < -tol, activate it and solve (B_a B_a^T + constraint_reg I) l = -c_u[a],
// dropping the active inequality whose multiplier first crosses zero on the
// segment from the previous multipliers until all are >= 0; then c = c_u +
// G[:, a] l (= B (y_u + B_a^T l) - t).  Stops when the active set did not
// change or after more than max_niter rounds; x = L^-T (y_u + B_a^T l).
//
// The reference refactors B_a B_a^T from scratch for every solve, its rows in
// constraint order.  Here the rows are kept in activation order and the
// factor grows by one row per activation (a forward substitution, O(a^2));
// removing row p recomputes rows p.. only.  The factor's first 48 rows (the
// active sets of multi-tissue CSD stay below the 47 parameters, in practice)
// live in shared memory, later rows in a per-warp global scratch.  The multipliers are the same
// (to rounding); ties in the choice of the constraint to drop still go to the
// lowest constraint index, as the reference's ascending scan does.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/csd_b200.h"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu
}

struct csd_icls {
  int nmeas = 0, nparam = 0, ncons = 0, num_eq = 0, max_niter = 0;
  double constraint_reg = 0.0, tol = 0.0;
  int device = 0;
  double* d_b2dT = nullptr;  // [nparam][nmeas]
  double* d_B = nullptr;     // [ncons][nparam]
  double* d_G = nullptr;     // [ncons][ncons]
  double* d_t = nullptr;     // [ncons] or null
  double* d_L = nullptr;     // [nparam][nparam], lower, row-major
  double* d_H = nullptr;     // [nmeas][nparam] (the predicted measurements H x)
  double* d_scratch = nullptr;  // per warp: the factor rows past the shared-memory part
  size_t scratch_warps = 0;
  char* d_host_ws = nullptr;  // csd_icls_solve_host's device staging, grown as needed
  size_t host_ws_bytes = 0;
  cudaStream_t host_stream = nullptr;
};

namespace {

constexpr int kIclsWarps = 4;  // warps per block
constexpr int kIclsMaxActive = 512;
constexpr int kIclsMaxParam = 256;
constexpr int kIclsSmemRows = 48;  // factor rows kept in shared memory (packed); later rows in global scratch
constexpr int kIclsSmemFactor = kIclsSmemRows * (kIclsSmemRows + 1) / 2;

// per-warp shared memory, in doubles: b, y_u, c_u, c, lam_prev, l, r (work,
// max(ncons, nparam)), inv (the factor's reciprocal diagonal), then act and
// pos (2 ncons ints in ncons doubles)
__host__ __device__ inline size_t icls_warp_doubles(int nmeas, int nparam, int ncons) {
  return (size_t)nmeas + nparam + 6 * (size_t)ncons + (size_t)(ncons > nparam ? ncons : nparam) + kIclsSmemFactor;
}

// Element (i, j <= i) of the active-set factor: rows below kIclsSmemRows
// packed in shared memory, later rows row-major in the warp's global scratch.
__device__ __forceinline__ double& lref(double* Ls, double* Lg, int ld, int i, int j) {
  return i < kIclsSmemRows ? Ls[i * (i + 1) / 2 + j] : Lg[(long long)i * ld + j];
}

struct IclsArgs {
  const float* b;
  const double* b64;  // FP64 right-hand sides instead of b (csd_icls_solve_f64)
  double* x64;        // FP64 solutions instead of x
  long long n, vs, ms;
  const uint8_t* mask;
  float* x;
  long long xs;
  int* niter;
  float* pred;
  long long ps;
  const double *b2dT, *B, *G, *t, *L, *H;
  double* scratch;
  int nmeas, nparam, ncons, num_eq, max_niter, ld;
  double reg, tol;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Appends row k of the active-set factor for constraint q: w = L^-1 S[k][0..k)
// by column-oriented forward substitution, L[k][k] = sqrt(S_kk - |w|^2), and
// extends z = L^-1 rhs by its new entry z_k = (rhs_q - w . z) / L[k][k].
__device__ __forceinline__ void factor_append(const IclsArgs& a, double* Ls, double* Lg, double* inv, double* r,
                                              double* z, const int* act, int k, int q, double rhs, int lane) {
  const double* Gq = a.G + (long long)q * a.ncons;
  for (int p = lane; p < k; p += 32) r[p] = Gq[act[p]];
  __syncwarp();
  for (int j = 0; j < k; ++j) {
    const double wj = r[j] * inv[j];
    __syncwarp();
    for (int i = j + 1 + lane; i < k; i += 32) r[i] -= lref(Ls, Lg, a.ld, i, j) * wj;
    if (lane == 0) r[j] = wj;
    __syncwarp();
  }
  double s = 0.0, t = 0.0;
  for (int p = lane; p < k; p += 32) {
    const double w = r[p];
    s = fma(w, w, s);
    t = fma(w, z[p], t);
    lref(Ls, Lg, a.ld, k, p) = w;
  }
  s = warp_sum(s);
  t = warp_sum(t);
  const double d = sqrt(Gq[q] + a.reg - s);
  if (lane == 0) {
    lref(Ls, Lg, a.ld, k, k) = d;
    inv[k] = 1.0 / d;
    z[k] = (rhs - t) / d;
  }
  __syncwarp();
}

// Removes row p of the na-row factor: Givens rotations of columns (c, c + 1),
// c = p .. na - 2, zero the diagonal of row c + 1 into column c (rows below
// rotated alike, and z with them: L z = rhs stays true without equation p);
// then rows p + 1.. move up one.
__device__ __forceinline__ void factor_remove(const IclsArgs& a, double* Ls, double* Lg, double* inv, double* z,
                                              int p, int na, int lane) {
  for (int c = p; c + 1 < na; ++c) {
    const int r0 = c + 1;
    const double x = lref(Ls, Lg, a.ld, r0, c), y = lref(Ls, Lg, a.ld, r0, r0);
    const double h = hypot(x, y);
    const double cs = x / h, sn = y / h;
    __syncwarp();
    for (int r = r0 + lane; r < na; r += 32) {
      double& u = lref(Ls, Lg, a.ld, r, c);
      double& v = lref(Ls, Lg, a.ld, r, c + 1);
      const double u0 = u, v0 = v;
      u = cs * u0 + sn * v0;
      v = cs * v0 - sn * u0;
    }
    if (lane == 0) {
      const double z0 = z[c], z1 = z[c + 1];
      z[c] = cs * z0 + sn * z1;
      z[c + 1] = cs * z1 - sn * z0;
      inv[c] = 1.0 / h;
    }
    __syncwarp();
  }
  // new row i (i >= p) = old row i + 1, columns 0..i (its column i + 1 is now 0)
  for (int i = p; i + 1 < na; ++i) {
    // (the two rows' storage does not overlap: packed row i ends where row i + 1 begins)
    for (int j = lane; j <= i; j += 32) lref(Ls, Lg, a.ld, i, j) = lref(Ls, Lg, a.ld, i + 1, j);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kIclsWarps * 32) icls_solve_kernel(const __grid_constant__ IclsArgs a) {
  extern __shared__ __align__(16) double ism_[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t wd = icls_warp_doubles(a.nmeas, a.nparam, a.ncons);
  double* bb = ism_ + warp * wd;
  double* yu = bb + a.nmeas;
  double* cu = yu + a.nparam;
  double* c = cu + a.ncons;
  double* lp = c + a.ncons;   // lambda_prev, by constraint
  double* z = lp + a.ncons;   // L^-1 (-c_u[act]), by active position
  double* r = z + a.ncons;    // work vector; the multipliers after a solve
  double* inv = r + (a.ncons > a.nparam ? a.ncons : a.nparam);  // 1 / diagonal of the factor
  double* Ls = inv + a.ncons;  // factor rows < kIclsSmemRows, packed
  int* act = reinterpret_cast<int*>(Ls + kIclsSmemFactor);  // active constraints, activation order
  int* pos = act + a.ncons;  // position of each constraint in act, -1 if inactive
  const long long gw = (long long)blockIdx.x * kIclsWarps + warp;
  const long long nw = (long long)gridDim.x * kIclsWarps;
  double* Lg = a.scratch + gw * (long long)a.ld * a.ld;  // factor rows >= kIclsSmemRows
  const int num_ineq = a.ncons - a.num_eq;
  for (long long v = gw; v < a.n; v += nw) {
    float* xo = a.x64 ? nullptr : a.x + v * a.xs;
    double* xo64 = a.x64 ? a.x64 + v * a.xs : nullptr;
    auto put = [&](int j, double val) {
      if (xo64)
        xo64[j] = val;
      else
        xo[j] = (float)val;
    };
    if (a.mask && !a.mask[v]) {
      for (int j = lane; j < a.nparam; j += 32) put(j, 0.0);
      if (a.pred)
        for (int i = lane; i < a.nmeas; i += 32) a.pred[v * a.ps + i] = 0.f;
      if (a.niter && lane == 0) a.niter[v] = 0;
      continue;
    }
    bool finite = true;
    for (int i = lane; i < a.nmeas; i += 32) {
      const long long o = v * a.vs + (long long)i * a.ms;
      const double f = a.b64 ? a.b64[o] : (double)a.b[o];
      finite &= isfinite(f);
      bb[i] = f;
    }
    if (!__all_sync(0xffffffffu, finite)) {
      // a non-finite measurement propagates through b2d^T b to every output
      for (int j = lane; j < a.nparam; j += 32) put(j, __longlong_as_double(0x7ff8000000000000ll));
      if (a.pred)
        for (int i = lane; i < a.nmeas; i += 32) a.pred[v * a.ps + i] = __int_as_float(0x7fffffff);
      if (a.niter && lane == 0) a.niter[v] = 0;
      continue;
    }
    __syncwarp();
    for (int j = lane; j < a.nparam; j += 32) {
      const double* w = a.b2dT + (long long)j * a.nmeas;
      double s = 0.0;
      for (int i = 0; i < a.nmeas; ++i) s = fma(w[i], bb[i], s);
      yu[j] = s;
    }
    __syncwarp();
    for (int m = lane; m < a.ncons; m += 32) {
      const double* w = a.B + (long long)m * a.nparam;
      double s = 0.0;
      for (int j = 0; j < a.nparam; ++j) s = fma(w[j], yu[j], s);
      if (a.t) s -= a.t[m];
      cu[m] = s;
      c[m] = s;
      lp[m] = 0.0;
      pos[m] = -1;
    }
    __syncwarp();
    int na = 0;           // active rows in the factor
    bool solved = false;  // r holds the multipliers of a solve (else x = y_u)
    // the equalities are active from the start (constrained_least_squares.h:265-266)
    for (int e = 0; e < a.num_eq; ++e) {
      const int q = num_ineq + e;
      if (lane == 0) {
        act[na] = q;
        pos[q] = na;
      }
      __syncwarp();
      factor_append(a, Ls, Lg, inv, r, z, act, na, q, -cu[q], lane);
      ++na;
    }
    int niter = 0;
    bool fail = false;
    while (num_ineq > 0) {
      // most violated inequality: lowest value, lowest index on ties
      double cmin = INFINITY;
      int imin = 0x7fffffff;
      for (int m = lane; m < num_ineq; m += 32)
        if (c[m] < cmin) {
          cmin = c[m];
          imin = m;
        }
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, cmin, o);
        const int oi = __shfl_xor_sync(0xffffffffu, imin, o);
        if (ov < cmin || (ov == cmin && oi < imin)) {
          cmin = ov;
          imin = oi;
        }
      }
      if (!(cmin < -a.tol)) break;
      bool changed = pos[imin] < 0;
      if (changed) {
        if (na >= a.ld) {
          fail = true;
          break;
        }
        if (lane == 0) {
          act[na] = imin;
          pos[imin] = na;
        }
        __syncwarp();
        factor_append(a, Ls, Lg, inv, r, z, act, na, imin, -cu[imin], lane);
        ++na;
      }
      while (true) {
        // the multipliers: L^T l = z by columns of L^T (rows of L)
        for (int p = lane; p < na; p += 32) r[p] = z[p];
        __syncwarp();
        for (int j = na - 1; j >= 0; --j) {
          const double lj = r[j] * inv[j];
          __syncwarp();
          for (int i = lane; i < j; i += 32) r[i] -= lref(Ls, Lg, a.ld, j, i) * lj;
          if (lane == 0) r[j] = lj;
          __syncwarp();
        }
        // the active inequality whose multiplier first crosses zero
        double smin = INFINITY;
        int sidx = 0x7fffffff, spos = -1;
        for (int p = lane; p < na; p += 32) {
          const int n = act[p];
          const double lv = r[p];
          if (n < num_ineq && lv < 0.0) {
            const double s = lp[n] / (lp[n] - lv);
            if (s < smin || (s == smin && n < sidx)) {
              smin = s;
              sidx = n;
              spos = p;
            }
          }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          const double ov = __shfl_xor_sync(0xffffffffu, smin, o);
          const int oi = __shfl_xor_sync(0xffffffffu, sidx, o);
          const int op = __shfl_xor_sync(0xffffffffu, spos, o);
          if (ov < smin || (ov == smin && oi < sidx)) {
            smin = ov;
            sidx = oi;
            spos = op;
          }
        }
        __syncwarp();
        if (!(smin < INFINITY)) {
          solved = true;
          break;
        }
        // drop it: rotate its row out of the factor, shift the later rows
        changed = true;
        factor_remove(a, Ls, Lg, inv, z, spos, na, lane);
        const int nact = na - 1;
        if (lane == 0) pos[sidx] = -1;
        for (int p0 = spos; p0 < nact; p0 += 32) {
          const int p = p0 + lane;
          const int q = p < nact ? act[p + 1] : 0;
          __syncwarp();
          if (p < nact) {
            act[p] = q;
            pos[q] = p;
          }
          __syncwarp();
        }
        __syncwarp();
        na = nact;
      }
      // lambda_prev: the new multipliers on the active inequalities, 0 elsewhere
      for (int m = lane; m < num_ineq; m += 32) lp[m] = pos[m] >= 0 ? r[pos[m]] : 0.0;
      __syncwarp();
      ++niter;
      if (!changed || niter > a.max_niter) break;
      for (int m = lane; m < a.ncons; m += 32) {
        double s = cu[m];
        for (int p = 0; p < na; ++p) s = fma(a.G[(long long)act[p] * a.ncons + m], r[p], s);
        c[m] = s;
      }
      __syncwarp();
    }
    if (fail) {
      for (int j = lane; j < a.nparam; j += 32) put(j, __longlong_as_double(0x7ff8000000000000ll));
      if (a.pred)
        for (int i = lane; i < a.nmeas; i += 32) a.pred[v * a.ps + i] = __int_as_float(0x7fffffff);
      if (a.niter && lane == 0) a.niter[v] = -1;
      continue;
    }
    // x = y_u + B_a^T l (into registers: r still holds l), then L^T z = x by
    // back substitution (rows of L)
    double xj[kIclsMaxParam / 32];
#pragma unroll
    for (int h = 0; h < kIclsMaxParam / 32; ++h) {
      const int j = lane + 32 * h;
      xj[h] = 0.0;
      if (j < a.nparam) {
        double s = yu[j];
        if (solved)
          for (int p = 0; p < na; ++p) s = fma(a.B[(long long)act[p] * a.nparam + j], r[p], s);
        xj[h] = s;
      }
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < kIclsMaxParam / 32; ++h)
      if (lane + 32 * h < a.nparam) r[lane + 32 * h] = xj[h];
    __syncwarp();
    for (int j = a.nparam - 1; j >= 0; --j) {
      const double zj = r[j] / a.L[(long long)j * a.nparam + j];
      __syncwarp();
      for (int i = lane; i < j; i += 32) r[i] -= a.L[(long long)j * a.nparam + i] * zj;
      if (lane == 0) r[j] = zj;
      __syncwarp();
    }
    for (int j = lane; j < a.nparam; j += 32) put(j, r[j]);
    if (a.pred)  // the predicted measurements H x (MSMT_Processor's -predicted_signal, dwi2fod.cpp:212-216)
      for (int i = lane; i < a.nmeas; i += 32) {
        const double* h = a.H + (long long)i * a.nparam;
        double s = 0.0;
        for (int j = 0; j < a.nparam; ++j) s = fma(h[j], r[j], s);
        a.pred[v * a.ps + i] = (float)s;
      }
    if (a.niter && lane == 0) a.niter[v] = niter;
    __syncwarp();
  }
}

// ---- host FP64 set-up ------------------------------------------------------

void cholesky_lower(std::vector<double>& S, int n) {  // in place, row-major, lower
  for (int j = 0; j < n; ++j) {
    double d = S[(size_t)j * n + j];
    for (int k = 0; k < j; ++k) d -= S[(size_t)j * n + k] * S[(size_t)j * n + k];
    if (!(d > 0.0)) throw std::runtime_error("ICLS problem matrix is not positive definite");
    d = std::sqrt(d);
    S[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = S[(size_t)i * n + j];
      for (int k = 0; k < j; ++k) s -= S[(size_t)i * n + k] * S[(size_t)j * n + k];
      S[(size_t)i * n + j] = s / d;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) S[(size_t)i * n + j] = 0.0;
}

// z = L^-1 v (forward substitution, L row-major lower)
void forward(const std::vector<double>& L, int n, const double* v, double* z) {
  for (int i = 0; i < n; ++i) {
    double s = v[i];
    for (int k = 0; k < i; ++k) s -= L[(size_t)i * n + k] * z[k];
    z[i] = s / L[(size_t)i * n + i];
  }
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src) {
  cudaError_t e = cudaMalloc(dst, src.size() * sizeof(T));
  if (e == cudaSuccess) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

namespace {
int icls_build(const double* H, bool standard, int nmeas, int nparam, const double* A, int ncons, const double* t,
               int num_eq, double solution_reg, double constraint_reg, int max_niter, double tol, csd_icls** out);
}

extern "C" int csd_icls_create(const double* H, int nmeas, int nparam, const double* A, int ncons, const double* t,
                               int num_eq, double solution_reg, double constraint_reg, int max_niter, double tol,
                               csd_icls** out) {
  return icls_build(H, false, nmeas, nparam, A, ncons, t, num_eq, solution_reg, constraint_reg, max_niter, tol, out);
}

extern "C" int csd_icls_create_standard(const double* HtH, int nparam, const double* A, int ncons, const double* t,
                                        int num_eq, double solution_reg, double constraint_reg, int max_niter,
                                        double tol, csd_icls** out) {
  return icls_build(HtH, true, nparam, nparam, A, ncons, t, num_eq, solution_reg, constraint_reg, max_niter, tol, out);
}

namespace {
int icls_build(const double* H, bool standard, int nmeas, int nparam, const double* A, int ncons, const double* t,
               int num_eq, double solution_reg, double constraint_reg, int max_niter, double tol, csd_icls** out) {
  if (!out || !H || !A || nmeas < 1 || nparam < 1 || ncons < 1 || num_eq < 0 || num_eq > ncons ||
      solution_reg < 0.0 || constraint_reg < 0.0 || tol < 0.0 || max_niter < 0 || ncons > 4096 || nparam > kIclsMaxParam ||
      nmeas > 4096 || num_eq > kIclsMaxActive)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_create: invalid argument");
  *out = nullptr;
  try {
    // H^T H (+ solution_reg * its largest diagonal entry) and its Cholesky factor
    std::vector<double> L((size_t)nparam * nparam, 0.0);
    for (int i = 0; i < nparam; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = 0.0;
        if (standard) {  // H^T H given (its lower triangle is read)
          s = H[(size_t)i * nparam + j];
        } else {
          for (int r = 0; r < nmeas; ++r) s += H[(size_t)r * nparam + i] * H[(size_t)r * nparam + j];
        }
        L[(size_t)i * nparam + j] = s;
      }
    double dmax = -INFINITY;
    for (int i = 0; i < nparam; ++i) dmax = std::max(dmax, L[(size_t)i * nparam + i]);
    for (int i = 0; i < nparam; ++i) L[(size_t)i * nparam + i] += solution_reg * dmax;
    cholesky_lower(L, nparam);
    // b2d^T = L^-1 H^T, B^T = L^-1 A^T (rows normalised)
    std::vector<double> b2dT((size_t)nparam * nmeas), B((size_t)ncons * nparam), tt, col(nparam), z(nparam);
    for (int r = 0; r < nmeas; ++r) {
      // b2d = H L^-T; in standard form the measurements are H^T b already: b2d = L^-T
      for (int i = 0; i < nparam; ++i) col[i] = standard ? (i == r ? 1.0 : 0.0) : H[(size_t)r * nparam + i];
      forward(L, nparam, col.data(), z.data());
      for (int i = 0; i < nparam; ++i) b2dT[(size_t)i * nmeas + r] = z[i];
    }
    if (t) tt.assign(t, t + ncons);
    for (int m = 0; m < ncons; ++m) {
      forward(L, nparam, A + (size_t)m * nparam, z.data());
      double nrm = 0.0;
      for (int i = 0; i < nparam; ++i) nrm += z[i] * z[i];
      nrm = std::sqrt(nrm);
      // a zero row normalises to NaN, as in the reference: its constraint
      // value is NaN, which the "most violated" scan never selects
      for (int i = 0; i < nparam; ++i) B[(size_t)m * nparam + i] = z[i] / nrm;
      if (t) tt[m] /= nrm;
    }
    std::vector<double> G((size_t)ncons * ncons);
    for (int i = 0; i < ncons; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = 0.0;
        for (int k = 0; k < nparam; ++k) s += B[(size_t)i * nparam + k] * B[(size_t)j * nparam + k];
        G[(size_t)i * ncons + j] = G[(size_t)j * ncons + i] = s;
      }
    auto* p = new csd_icls();
    p->nmeas = nmeas;
    p->nparam = nparam;
    p->ncons = ncons;
    p->num_eq = num_eq;
    p->max_niter = max_niter ? max_niter : 10 * nparam;
    p->constraint_reg = constraint_reg;
    p->tol = tol;
    cudaError_t e = cudaGetDevice(&p->device);
    if (e == cudaSuccess) e = upload(&p->d_b2dT, b2dT);
    if (e == cudaSuccess) e = upload(&p->d_B, B);
    if (e == cudaSuccess) e = upload(&p->d_G, G);
    if (e == cudaSuccess) e = upload(&p->d_L, L);
    if (e == cudaSuccess && !standard) e = upload(&p->d_H, std::vector<double>(H, H + (size_t)nmeas * nparam));
    if (e == cudaSuccess && t) e = upload(&p->d_t, tt);
    if (e != cudaSuccess) {
      csd_icls_destroy(p);
      return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_create: ") + cudaGetErrorString(e));
    }
    *out = p;
  } catch (const std::exception& ex) {
    return csdb200::set_error(CSD_ERR_INVALID, std::string("csd_icls_create: ") + ex.what());
  }
  return CSD_OK;
}

}  // namespace

extern "C" void csd_icls_destroy(csd_icls* p) {
  if (!p) return;
  cudaFree(p->d_b2dT);
  cudaFree(p->d_B);
  cudaFree(p->d_G);
  cudaFree(p->d_t);
  cudaFree(p->d_L);
  cudaFree(p->d_H);
  cudaFree(p->d_scratch);
  cudaFree(p->d_host_ws);
  if (p->host_stream) cudaStreamDestroy(p->host_stream);
  delete p;
}

extern "C" int csd_icls_info(const csd_icls* p, int* out4) {
  if (!p || !out4) return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_info: invalid argument");
  out4[0] = p->nmeas;
  out4[1] = p->nparam;
  out4[2] = p->ncons;
  out4[3] = p->max_niter;
  return CSD_OK;
}

namespace {
int icls_solve(csd_icls* p, const float* b, const double* b64, int64_t n, int64_t voxel_stride, int64_t meas_stride,
               const uint8_t* mask, float* x, double* x64, int64_t x_stride, int32_t* niter, float* pred,
               int64_t pred_stride, void* stream);
}

extern "C" int csd_icls_solve(csd_icls* p, const float* b, int64_t n, int64_t voxel_stride, int64_t meas_stride,
                              const uint8_t* mask, float* x, int64_t x_stride, int32_t* niter, float* pred,
                              int64_t pred_stride, void* stream) {
  if (!p || n < 0 || (n > 0 && (!b || !x)))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_solve: invalid argument");
  return icls_solve(p, b, nullptr, n, voxel_stride, meas_stride, mask, x, nullptr, x_stride, niter, pred, pred_stride,
                    stream);
}

extern "C" int csd_icls_solve_f64(csd_icls* p, const double* b, int64_t n, int64_t voxel_stride, int64_t meas_stride,
                                  double* x, int64_t x_stride, int32_t* niter, void* stream) {
  if (!p || n < 0 || (n > 0 && (!b || !x)))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_solve_f64: invalid argument");
  return icls_solve(p, nullptr, b, n, voxel_stride, meas_stride, nullptr, nullptr, x, x_stride, niter, nullptr, 0,
                    stream);
}

namespace {
int icls_solve(csd_icls* p, const float* b, const double* b64, int64_t n, int64_t voxel_stride, int64_t meas_stride,
               const uint8_t* mask, float* x, double* x64, int64_t x_stride, int32_t* niter, float* pred,
               int64_t pred_stride, void* stream) {
  if (x_stride < p->nparam || (pred && (pred_stride < p->nmeas || !p->d_H)))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_solve: invalid argument (predicted measurements need a "
                                               "problem given by H)");
  if (n == 0) return CSD_OK;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int nsm = 0, smem_max = 0;
  cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_solve: ") + cudaGetErrorString(e));
  const size_t smem = kIclsWarps * icls_warp_doubles(p->nmeas, p->nparam, p->ncons) * sizeof(double);
  if (smem > (size_t)smem_max)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_solve: problem too large for shared memory");
  e = cudaFuncSetAttribute(icls_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, icls_solve_kernel, kIclsWarps * 32, smem);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_solve: ") + cudaGetErrorString(e));
  const long long blocks = std::max<long long>(
      1, std::min<long long>((n + kIclsWarps - 1) / kIclsWarps, (long long)nsm * std::max(1, per_sm)));
  const int ld = std::min(p->ncons, kIclsMaxActive);
  const size_t warps = (size_t)blocks * kIclsWarps;
  if (warps > p->scratch_warps) {
    // each warp's factor rows beyond the shared-memory part (row-major, ld)
    cudaFree(p->d_scratch);
    p->d_scratch = nullptr;
    p->scratch_warps = 0;
    e = cudaMalloc(&p->d_scratch, warps * (size_t)ld * ld * sizeof(double));
    if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_solve: ") + cudaGetErrorString(e));
    p->scratch_warps = warps;
  }
  IclsArgs a{};
  a.b = b;
  a.b64 = b64;
  a.x64 = x64;
  a.n = n;
  a.vs = voxel_stride;
  a.ms = meas_stride;
  a.mask = mask;
  a.x = x;
  a.xs = x_stride;
  a.niter = niter;
  a.pred = pred;
  a.ps = pred_stride;
  a.H = p->d_H;
  a.b2dT = p->d_b2dT;
  a.B = p->d_B;
  a.G = p->d_G;
  a.t = p->d_t;
  a.L = p->d_L;
  a.scratch = p->d_scratch;
  a.nmeas = p->nmeas;
  a.nparam = p->nparam;
  a.ncons = p->ncons;
  a.num_eq = p->num_eq;
  a.max_niter = p->max_niter;
  a.ld = ld;
  a.reg = p->constraint_reg;
  a.tol = p->tol;
  {
    icls_solve_kernel<<<(unsigned)blocks, kIclsWarps * 32, smem, st>>>(a);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_solve: ") + cudaGetErrorString(e));
  return CSD_OK;
}

}  // namespace

// The solver on HOST buffers (b [n][voxel_stride] float, x [n][nparam],
// niter / mask / pred optional): device staging (kept with the problem for
// later calls, with its stream), one solve, copies back; synchronous.  The solve dominates (milliseconds per thousand voxels against
// microseconds of transfer), so the copies are not overlapped.
extern "C" int csd_icls_solve_host(csd_icls* p, const float* b, int64_t n, int64_t voxel_stride,
                                   const uint8_t* mask, float* x, int32_t* niter, float* pred) {
  if (!p || n < 0 || (n > 0 && (!b || !x)) || voxel_stride < p->nmeas)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_icls_solve_host: invalid argument");
  if (n == 0) return CSD_OK;
  const size_t nb = (size_t)n * voxel_stride * sizeof(float), nx = (size_t)n * p->nparam * sizeof(float);
  const size_t np = pred ? (size_t)n * p->nmeas * sizeof(float) : 0, nm = mask ? (size_t)n : 0;
  const size_t off_x = (nb + 255) / 256 * 256, off_i = off_x + (nx + 255) / 256 * 256,
               off_p = off_i + ((size_t)n * sizeof(int32_t) + 255) / 256 * 256,
               off_m = off_p + (np + 255) / 256 * 256, total = off_m + nm;
  cudaError_t e = cudaSuccess;
  if (total > p->host_ws_bytes) {  // the staging buffer is kept for later calls
    cudaFree(p->d_host_ws);
    p->d_host_ws = nullptr;
    p->host_ws_bytes = 0;
    e = cudaMalloc(&p->d_host_ws, total);
    if (e != cudaSuccess)
      return csdb200::set_error(CSD_ERR_NOMEM, std::string("csd_icls_solve_host: ") + cudaGetErrorString(e));
    p->host_ws_bytes = total;
  }
  if (!p->host_stream) e = cudaStreamCreateWithFlags(&p->host_stream, cudaStreamNonBlocking);
  char* d = p->d_host_ws;
  cudaStream_t st = p->host_stream;
  if (e == cudaSuccess) e = cudaMemcpyAsync(d, b, nb, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && mask) e = cudaMemcpyAsync(d + off_m, mask, nm, cudaMemcpyHostToDevice, st);
  int rc = CSD_OK;
  if (e == cudaSuccess)
    rc = csd_icls_solve(p, reinterpret_cast<const float*>(d), n, voxel_stride, 1,
                        mask ? reinterpret_cast<const uint8_t*>(d + off_m) : nullptr, reinterpret_cast<float*>(d + off_x),
                        p->nparam, reinterpret_cast<int32_t*>(d + off_i), pred ? reinterpret_cast<float*>(d + off_p) : nullptr,
                        p->nmeas, st);
  if (e == cudaSuccess && rc == CSD_OK) e = cudaMemcpyAsync(x, d + off_x, nx, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && rc == CSD_OK && niter)
    e = cudaMemcpyAsync(niter, d + off_i, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && rc == CSD_OK && pred) e = cudaMemcpyAsync(pred, d + off_p, np, cudaMemcpyDeviceToHost, st);
  if (st) {
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
  }
  if (rc != CSD_OK) return rc;
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_icls_solve_host: ") + cudaGetErrorString(e));
  return CSD_OK;
}
