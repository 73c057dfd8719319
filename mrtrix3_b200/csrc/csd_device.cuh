// Device-side building blocks of single-shell CSD for sm_100a.
//
// One warp owns one voxel at a time and runs MRtrix3's per-voxel algorithm
// (src/dwi/sdeconv/csd.h:237-269) on it:
//   set      F = [rconv S; 0], b = M^T S                       (csd.h:237-243)
//   project  a = HR_trans F, neg = {d : a_d < threshold}        (csd.h:246-250)
//   compare  stop when neg equals the previous set              (csd.h:252-253)
//   assemble W = Mt_M + HR_trans[neg]^T HR_trans[neg]           (csd.h:255-262)
//   solve    F = W^-1 b by Cholesky                             (csd.h:264)
// Numerics: projection, assembly, factorisation and substitutions in FP32;
// one refinement step whose residual b - W F is accumulated in FP64; a
// factorisation is redone in FP64 when its pivots fail or the condition
// estimate (max L_ii / min L_ii)^2 exceeds a threshold.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace csdb200 {

constexpr int kMaxHR = 512;          // constraint directions supported
constexpr int kMaxDW = 512;          // DW volumes in the selected shell supported
constexpr int kMaxWords = kMaxHR / 32;
constexpr int kMaxVolumesPerLaunch = 48;

// Packed lower-triangular storage with every row padded to a multiple of 4
// floats so rows can be read as float4: row i starts at packoff(i).
__host__ __device__ constexpr int packoff(int i) {
  return 4 * (i + 2 * (i >> 2) * ((i >> 2) - 1) + (i & 3) * (i >> 2));
}
// Row stride of the constraint matrix in shared memory: a multiple of 4 whose
// float4 count is odd, so lanes reading different rows hit distinct banks.
__host__ __device__ constexpr int hr_stride(int n) {
  return (((n + 3) / 4) % 2 == 1) ? ((n + 3) / 4) * 4 : ((n + 3) / 4 + 1) * 4;
}

template <int N>
struct Dims {
  static constexpr int CQ = (N + 31) / 32;        // coefficient slots per lane
  static constexpr int HS = hr_stride(N);         // HR row stride (floats)
  static constexpr int WSZ = packoff(N);          // packed W size (floats)
  static constexpr int NB = (N + 3) / 4;          // 4-row blocks
  static constexpr int NBLK = NB * (NB + 1) / 2;  // lower-triangle blocks
  static constexpr int BPL = (NBLK + 31) / 32;    // blocks per lane
  static constexpr int GROUP = 3;                 // blocks accumulated per pass
  static constexpr int PASSES = (BPL + GROUP - 1) / GROUP;
  // threads per block of the persistent kernel (bounds the register budget)
  static constexpr int THREADS = N <= 45 ? 512 : (N <= 66 ? 384 : 192);
};

// Everything a voxel of one image needs, by device pointer.
struct Scheme {
  const float* H32;       // [nhr][HS] HR_trans, fp32, zero padded
  const double* H64;      // [nhr][nsh] HR_trans, fp64 (FP64 fallback)
  const float* MtMp;      // packed-padded lower Mt_M, fp32
  const double* MtM64;    // [nsh][nsh] full Mt_M, fp64 (refinement residual)
  const double* rconvT;   // [ndw][ninit] rconv^T, fp64
  const double* M64;      // [ndw][nsh] M, fp64
  const int* dwis;        // [ndw]
  int ndw, ninit, niter;
  float threshold;
};

struct VolumeDesc {
  Scheme sc;
  const float* dwi;
  long long n_voxels, vox_stride, vol_stride, first;  // first = global index of voxel 0
  const uint8_t* mask;
  const uint32_t* warm;
  float* fod;
  long long fod_stride;
  uint8_t* status;
  uint8_t* iters;
  uint32_t* negmask;
};

struct SolveParams {
  int n_vol, nhr, nw, refine;
  float cond_thr;
  long long total;
  unsigned long long* queue;     // work counter, zeroed before launch
  double* fp64_scratch;          // [gridDim.x * warps][WSZ] doubles
  VolumeDesc vol[kMaxVolumesPerLaunch];
};

// Per-warp shared-memory workspace (carved from dynamic shared memory).
template <int N>
__host__ __device__ constexpr int wbuf_floats() {
  return Dims<N>::WSZ > kMaxDW ? Dims<N>::WSZ : kMaxDW;
}

template <int N>
struct WarpWS {
  float* W;        // [WSZ] packed W / L (also holds S during set)
  float* F;        // [HS] current F (fp32)
  double* b;       // [N] M^T S (fp64)
  uint16_t* neg;   // [kMaxHR] negative-set index list
};

template <int N>
__host__ __device__ constexpr int warp_ws_bytes() {
  return wbuf_floats<N>() * 4 + Dims<N>::HS * 4 + ((N * 8 + 15) / 16) * 16 + kMaxHR * 2;
}

template <int N>
__device__ __forceinline__ WarpWS<N> carve_ws(unsigned char* base) {
  WarpWS<N> w;
  w.W = reinterpret_cast<float*>(base);
  w.F = w.W + wbuf_floats<N>();
  w.b = reinterpret_cast<double*>(w.F + Dims<N>::HS);
  w.neg = reinterpret_cast<uint16_t*>(reinterpret_cast<unsigned char*>(w.b) + ((N * 8 + 15) / 16) * 16);
  return w;
}

__device__ __forceinline__ double shfl_d(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// ---------------------------------------------------------------------------
// set(): load + clamp the voxel's DW samples (dwi2fod.cpp:156-173), then
// F = [rconv S; 0] and b = M^T S (csd.h:237-243), both accumulated in FP64.
// Returns 0 = ok, 1 = masked out, 3 = non-finite sample.
template <int N>
__device__ int voxel_set(const Scheme& sc, const float* dwi, long long vol_stride, bool masked,
                         const WarpWS<N>& w, int lane) {
  if (masked) return 1;
  float* S = w.W;  // W is free during set
  bool bad = false;
  for (int t = lane; t < sc.ndw; t += 32) {
    float v = __ldg(dwi + (long long)__ldg(sc.dwis + t) * vol_stride);
    if (!isfinite(v)) bad = true;
    S[t] = v < 0.f ? 0.f : v;
  }
  if (__any_sync(0xffffffffu, bad)) return 3;
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int c = lane + 32 * q;
    double f = 0.0, bb = 0.0;
    if (c < N) {
      for (int t = 0; t < sc.ndw; ++t) {
        const double s = (double)S[t];
        if (c < sc.ninit) f = fma(__ldg(sc.rconvT + (long long)t * sc.ninit + c), s, f);
        bb = fma(__ldg(sc.M64 + (long long)t * N + c), s, bb);
      }
      w.b[c] = bb;
    }
    if (c < Dims<N>::HS) w.F[c] = (c < N) ? (float)f : 0.f;
  }
  for (int c = lane + 32 * Dims<N>::CQ; c < Dims<N>::HS; c += 32) w.F[c] = 0.f;
  __syncwarp();
  return 0;
}

// ---------------------------------------------------------------------------
// Projection onto the constraint directions and the negative-set bitmask
// (csd.h:246-250).  Lane l evaluates directions l, l+32, ...; the F vector is
// read as broadcast float4s, HR rows as float4s (conflict-free stride).
template <int N>
__device__ __forceinline__ void project_mask(const float* Hs, int nhr, int nw, float thr,
                                             const WarpWS<N>& w, int lane, uint32_t* bits) {
  constexpr int HS = Dims<N>::HS;
  float acc[kMaxWords];
#pragma unroll
  for (int p = 0; p < kMaxWords; ++p) acc[p] = 0.f;
#pragma unroll 4
  for (int j = 0; j < HS / 4; ++j) {
    const float4 f4 = reinterpret_cast<const float4*>(w.F)[j];
#pragma unroll
    for (int p = 0; p < kMaxWords; ++p) {
      if (p < nw) {
        const int d = lane + 32 * p;
        if (d < nhr) {
          const float4 h4 = reinterpret_cast<const float4*>(Hs + d * HS)[j];
          acc[p] = fmaf(h4.x, f4.x, acc[p]);
          acc[p] = fmaf(h4.y, f4.y, acc[p]);
          acc[p] = fmaf(h4.z, f4.z, acc[p]);
          acc[p] = fmaf(h4.w, f4.w, acc[p]);
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < kMaxWords; ++p) {
    if (p < nw) {
      const int d = lane + 32 * p;
      bits[p] = __ballot_sync(0xffffffffu, d < nhr && acc[p] < thr);
    }
  }
}

// Expand a bitmask into the ordered index list HR_T's rows are gathered from
// (csd.h:257-259).  Returns k = |neg|.
__device__ __forceinline__ int mask_to_list(const uint32_t* bits, int nw, uint16_t* neg, int lane) {
  int k = 0;
#pragma unroll
  for (int p = 0; p < kMaxWords; ++p) {
    if (p < nw) {
      const uint32_t m = bits[p];
      if ((m >> lane) & 1u) neg[k + __popc(m & ((1u << lane) - 1u))] = (uint16_t)(32 * p + lane);
      k += __popc(m);
    }
  }
  __syncwarp();
  return k;
}

// ---------------------------------------------------------------------------
// W = Mt_M + sum_{d in neg} h_d h_d^T, lower triangle (csd.h:255-262).
// Each lane owns up to 3 4x4 blocks of the lower triangle per pass and keeps
// them in registers while streaming over the gathered rows.
template <int N>
__device__ void assemble(const float* Hs, const float* MtMp, int k, const WarpWS<N>& w, int lane) {
  using D = Dims<N>;
#pragma unroll 1
  for (int pass = 0; pass < D::PASSES; ++pass) {
    int bi[D::GROUP], bj[D::GROUP];
    bool valid[D::GROUP];
    float acc[D::GROUP][16];
#pragma unroll
    for (int g = 0; g < D::GROUP; ++g) {
      const int b = lane + 32 * (pass * D::GROUP + g);
      valid[g] = b < D::NBLK;
      // invert b = bi (bi + 1) / 2 + bj
      int r = (int)((sqrtf(8.f * (float)b + 1.f) - 1.f) * 0.5f);
      while ((r + 1) * (r + 2) / 2 <= b) ++r;
      while (r * (r + 1) / 2 > b) --r;
      bi[g] = valid[g] ? r : 0;
      bj[g] = valid[g] ? b - r * (r + 1) / 2 : 0;
#pragma unroll
      for (int e = 0; e < 16; ++e) acc[g][e] = 0.f;
    }
#pragma unroll 2
    for (int q = 0; q < k; ++q) {
      const float4* h = reinterpret_cast<const float4*>(Hs + (int)w.neg[q] * D::HS);
#pragma unroll
      for (int g = 0; g < D::GROUP; ++g) {
        if (valid[g]) {
          const float4 a = h[bi[g]];
          const float4 c = h[bj[g]];
          const float av[4] = {a.x, a.y, a.z, a.w};
          const float cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
          for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int s = 0; s < 4; ++s) acc[g][r * 4 + s] = fmaf(av[r], cv[s], acc[g][r * 4 + s]);
        }
      }
    }
#pragma unroll
    for (int g = 0; g < D::GROUP; ++g) {
      if (valid[g]) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int i = 4 * bi[g] + r;
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            const int j = 4 * bj[g] + s;
            if (i < N && j <= i) {
              const int o = packoff(i) + j;
              w.W[o] = __ldg(MtMp + o) + acc[g][r * 4 + s];
            }
          }
        }
      }
    }
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// In-place left-looking Cholesky of the packed-padded lower matrix A (shared
// or global memory).  Lane l computes rows j+l, j+l+32, ... of column j.
// Returns false if a pivot is not positive; dmin/dmax receive the range of
// the diagonal of L.
template <int N, typename T>
__device__ bool cholesky_packed(T* A, int lane, T& dmin, T& dmax) {
  dmin = (T)1.0e300;
  dmax = (T)0;
  bool ok = true;
#pragma unroll 1
  for (int j = 0; j < N; ++j) {
    const T* Lj = A + packoff(j);
    T s[Dims<N>::CQ];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j + lane + 32 * q;
      s[q] = 0;
      if (i < N) {
        const T* Li = A + packoff(i);
        T acc = Li[j];
        for (int kk = 0; kk < j; ++kk) acc -= Li[kk] * Lj[kk];
        s[q] = acc;
      }
    }
    const T djj = __shfl_sync(0xffffffffu, s[0], 0);
    if (!(djj > (T)0)) {
      ok = false;
      break;
    }
    const T d = sqrt(djj);
    dmin = d < dmin ? d : dmin;
    dmax = d > dmax ? d : dmax;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j + lane + 32 * q;
      if (i < N) A[packoff(i) + j] = (i == j) ? d : s[q] / d;
    }
    __syncwarp();
  }
  __syncwarp();
  return ok;
}

// float specialisation with float4 row reads for the dot products
template <int N>
__device__ bool cholesky_packed_f32(float* A, int lane, float& dmin, float& dmax) {
  dmin = 3.0e38f;
  dmax = 0.f;
#pragma unroll 1
  for (int j = 0; j < N; ++j) {
    const float* Lj = A + packoff(j);
    const int j4 = j & ~3;
    float s[Dims<N>::CQ];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j + lane + 32 * q;
      s[q] = 0.f;
      if (i < N) {
        const float* Li = A + packoff(i);
        float a0 = 0.f, a1 = 0.f;
        for (int kk = 0; kk < j4; kk += 4) {
          const float4 x = *reinterpret_cast<const float4*>(Li + kk);
          const float4 y = *reinterpret_cast<const float4*>(Lj + kk);
          a0 = fmaf(x.x, y.x, a0);
          a1 = fmaf(x.y, y.y, a1);
          a0 = fmaf(x.z, y.z, a0);
          a1 = fmaf(x.w, y.w, a1);
        }
        for (int kk = j4; kk < j; ++kk) a0 = fmaf(Li[kk], Lj[kk], a0);
        s[q] = Li[j] - (a0 + a1);
      }
    }
    const float djj = __shfl_sync(0xffffffffu, s[0], 0);
    if (!(djj > 0.f) || !isfinite(djj)) return false;
    const float d = sqrtf(djj);
    dmin = fminf(dmin, d);
    dmax = fmaxf(dmax, d);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j + lane + 32 * q;
      if (i < N) A[packoff(i) + j] = (i == j) ? d : s[q] / d;
    }
    __syncwarp();
  }
  return true;
}

// x := L^-T L^-1 x with x distributed as x[q] = element lane + 32 q.
template <int N, typename T, typename LT>
__device__ __forceinline__ void chol_subst(const LT* L, T* x, int lane) {
  // forward: column sweep
#pragma unroll 1
  for (int kk = 0; kk < N; ++kk) {
    const int src = kk & 31, slot = kk >> 5;
    T xv = 0;
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q)
      if (q == slot) xv = x[q];
    const T xk = __shfl_sync(0xffffffffu, xv, src) / (T)L[packoff(kk) + kk];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i > kk && i < N) x[q] -= (T)L[packoff(i) + kk] * xk;
      if (i == kk) x[q] = xk;
    }
  }
  // backward with L^T: row kk of L holds column kk of L^T
#pragma unroll 1
  for (int kk = N - 1; kk >= 0; --kk) {
    const int src = kk & 31, slot = kk >> 5;
    T xv = 0;
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q)
      if (q == slot) xv = x[q];
    const T xk = __shfl_sync(0xffffffffu, xv, src) / (T)L[packoff(kk) + kk];
    const LT* Lk = L + packoff(kk);
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < kk) x[q] -= (T)Lk[i] * xk;
      if (i == kk) x[q] = xk;
    }
  }
}

// r = b - (Mt_M F + sum_{d in neg} h_d (h_d . F)), accumulated in FP64 with
// the FP32 operators the solve used.  F is read from w.F.
template <int N>
__device__ void residual_fp64(const Scheme& sc, const float* Hs, int k, const WarpWS<N>& w, int lane,
                              double* r) {
  constexpr int HS = Dims<N>::HS;
  double u[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) u[q] = 0.0;
  for (int q0 = 0; q0 < k; q0 += 32) {
    const int qq = q0 + lane;
    double t = 0.0;
    if (qq < k) {
      const float4* h = reinterpret_cast<const float4*>(Hs + (int)w.neg[qq] * HS);
      const float4* f = reinterpret_cast<const float4*>(w.F);
#pragma unroll 4
      for (int j = 0; j < HS / 4; ++j) {
        const float4 a = h[j], c = f[j];
        t = fma((double)a.x, (double)c.x, t);
        t = fma((double)a.y, (double)c.y, t);
        t = fma((double)a.z, (double)c.z, t);
        t = fma((double)a.w, (double)c.w, t);
      }
    }
    const int cnt = min(32, k - q0);
    for (int s = 0; s < cnt; ++s) {
      const double ts = shfl_d(t, s);
      const float* h = Hs + (int)w.neg[q0 + s] * HS;
#pragma unroll
      for (int q = 0; q < Dims<N>::CQ; ++q) {
        const int i = lane + 32 * q;
        if (i < N) u[q] = fma(ts, (double)h[i], u[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    double acc = 0.0;
    if (i < N) {
      const double* Mi = sc.MtM64 + (long long)i * N;
      for (int c = 0; c < N; ++c) acc = fma(__ldg(Mi + c), (double)w.F[c], acc);
      r[q] = w.b[i] - (acc + u[q]);
    } else {
      r[q] = 0.0;
    }
  }
}

// FP64 rebuild + factorisation + solve of the current system into w.F,
// used when the FP32 factorisation fails or is ill-conditioned.  Returns
// false if the FP64 factorisation fails as well.
template <int N>
__device__ bool solve_fp64(const Scheme& sc, int k, const WarpWS<N>& w, double* A, int lane) {
#pragma unroll 1
  for (int i = 0; i < N; ++i) {
    for (int j = lane; j <= i; j += 32) {
      double acc = 0.0;
      for (int q = 0; q < k; ++q) {
        const double* h = sc.H64 + (long long)w.neg[q] * N;
        acc = fma(__ldg(h + i), __ldg(h + j), acc);
      }
      A[packoff(i) + j] = __ldg(sc.MtM64 + (long long)i * N + j) + acc;
    }
  }
  __syncwarp();
  __threadfence_block();
  double dmin, dmax;
  const bool ok = cholesky_packed<N, double>(A, lane, dmin, dmax);
  double x[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    x[q] = i < N ? w.b[i] : 0.0;
  }
  if (ok) chol_subst<N, double, double>(A, x, lane);
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    if (i < N) w.F[i] = ok ? (float)x[q] : w.F[i];
  }
  __syncwarp();
  return ok;
}

// One assemble + factorise + solve (+ refinement) for the set in w.neg[0..k).
// Returns status flags (CSD_STATUS_FP64 / CSD_STATUS_CHOLFAIL bits).
template <int N>
__device__ int assemble_solve(const Scheme& sc, const float* Hs, int k, const WarpWS<N>& w, int lane,
                              float cond_thr, int refine, double* fp64_slot) {
  assemble<N>(Hs, sc.MtMp, k, w, lane);
  float dmin, dmax;
  const bool ok = cholesky_packed_f32<N>(w.W, lane, dmin, dmax);
  const float cond = ok ? (dmax / dmin) * (dmax / dmin) : 3.0e38f;
  if (!ok || !(cond <= cond_thr)) {
    const bool ok64 = solve_fp64<N>(sc, k, w, fp64_slot, lane);
    return 0x10 | (ok64 ? 0 : 0x20);
  }
  float x[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    x[q] = i < N ? (float)w.b[i] : 0.f;
  }
  chol_subst<N, float, float>(w.W, x, lane);
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    if (i < N) w.F[i] = x[q];
  }
  __syncwarp();
  if (refine) {
    double r[Dims<N>::CQ];
    residual_fp64<N>(sc, Hs, k, w, lane, r);
    float d[Dims<N>::CQ];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) d[q] = (float)r[q];
    chol_subst<N, float, float>(w.W, d, lane);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < N) w.F[i] = x[q] + d[q];
    }
    __syncwarp();
  }
  return 0;
}

}  // namespace csdb200
