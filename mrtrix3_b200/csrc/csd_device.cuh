// Device-side building blocks of single-shell CSD for sm_100a.
//
// One warp owns one voxel at a time and runs MRtrix3's per-voxel algorithm
// (src/dwi/sdeconv/csd.h:237-269) on it:
//   set      F = [rconv S; 0], b = M^T S                       (csd.h:237-243)
//   project  a = HR_trans F, neg = {d : a_d < threshold}        (csd.h:246-250)
//   compare  stop when neg equals the previous set              (csd.h:252-253)
//   assemble W = Mt_M + HR_trans[neg]^T HR_trans[neg]           (csd.h:255-262)
//   solve    F = W^-1 b by Cholesky                             (csd.h:264)
// Numerics:
//   * projection in FP32 (FP32 HR_trans, or its FP16 hi+lo pair re-summed);
//   * the rank-k assembly on the tensor cores with mma.sync m16n8k16: HR_trans
//     is split into FP16 hi + lo (22 significant bits) and W accumulates
//     hi*hi + hi*lo + lo*hi in FP32; the gathered rows are read straight from
//     the shared-memory table by ldmatrix row addresses (no gather copy);
//   * Cholesky and substitutions in FP32;
//   * one refinement step whose residual b - W F is accumulated in FP64
//     against the FP32 operator -- applied once the negative set repeats
//     (the fixed-point check is then repeated on the refined F), or after
//     every solve, or never, or (the default) after every solve of a voxel
//     whose negative set has come back after one step, i.e. cycles in FP32
//     (SolveParams::refine = 2 / 1 / 0 / 3);
//   * a factorisation is redone in FP64 when a pivot fails or the condition
//     estimate (max L_ii / min L_ii)^2 exceeds a threshold.
#pragma once

#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace csdb200 {

// Optional per-phase cycle counters (build with -DCSD_PHASE_TIMERS): each
// warp accumulates clock64() deltas per phase and adds them to
// g_phase_cycles at the end of the launch.  Off in the normal build.
#ifdef CSD_PHASE_TIMERS
__device__ unsigned long long g_phase_cycles[16];
#define CSD_T0(var) long long var = clock64()
#define CSD_T1(acc, idx, var) acc[idx] += clock64() - var
#else
#define CSD_T0(var)
#define CSD_T1(acc, idx, var)
#endif
enum Phase { kPhSet = 0, kPhProject, kPhAssemble, kPhChol, kPhSubst, kPhRefine, kPhFp64, kPhList, kPhTotal };

constexpr int kMaxHR = 512;          // constraint directions supported
constexpr int kMaxDW = 512;          // DW volumes in the selected shell supported
constexpr int kMaxWords = kMaxHR / 32;
constexpr int kMaxVolumesPerLaunch = 48;

// Packed lower-triangular storage with every row padded to a multiple of 4
// floats so rows can be read as float4: row i starts at packoff(i).
// Loop shapes of the FP32 factorisation and back substitution: the column
// blocks are unrolled, so every block's row offsets, trip counts and edge
// tests are compile-time constants (the integer and branch instructions
// around the arithmetic were half of the solve kernel's instructions); the
// factorisation's inner dot-product loop stays rolled to bound code size
// and registers.  Overridable for experiments.
#ifndef CSD_CHOL_CB_PRAGMA
#define CSD_CHOL_CB_PRAGMA _Pragma("unroll")
#endif
#ifndef CSD_CHOL_KK_PRAGMA
#define CSD_CHOL_KK_PRAGMA _Pragma("unroll 1")
#endif
#ifndef CSD_BACK_CB_PRAGMA
#ifdef CSD_BACK_ROLLED
#define CSD_BACK_CB_PRAGMA _Pragma("unroll 1")
#else
#define CSD_BACK_CB_PRAGMA _Pragma("unroll")
#endif
#endif
__host__ __device__ constexpr int packoff(int i) {
  return 4 * (i + 2 * (i >> 2) * ((i >> 2) - 1) + (i & 3) * (i >> 2));
}
// Row stride of the FP32 constraint matrix in shared memory: a multiple of 4
// whose float4 count is odd, so lanes reading different rows hit distinct banks.
__host__ __device__ constexpr int hr_stride(int n) {
  return (((n + 3) / 4) % 2 == 1) ? ((n + 3) / 4) * 4 : ((n + 3) / 4 + 1) * 4;
}
// Row stride (halves) of the FP16 hi/lo tables: covers 16-column blocks and
// has an odd number of 16-byte chunks (spreads ldmatrix rows over banks).
__host__ __device__ constexpr int hr_stride16(int n) {
  return ((((n + 15) / 16) * 16 / 8) % 2 == 1) ? ((n + 15) / 16) * 16 : ((n + 15) / 16) * 16 + 8;
}

template <int N>
struct Dims {
  static constexpr int CQ = (N + 31) / 32;        // coefficient slots per lane
  static constexpr int HS = hr_stride(N);         // FP32 HR row stride (floats)
  static constexpr int HS16 = hr_stride16(N);     // FP16 HR row stride (halves)
  static constexpr int NQ = (N + 3) / 4;          // float4 quads per row
  static constexpr int WSZ = packoff(N);          // packed W size (floats)
  static constexpr int NRB = (N + 15) / 16;       // 16-row blocks of W
  static constexpr int NJB = (N + 7) / 8;         // 8-column blocks of W
  static constexpr bool KEEP32 = N <= 45;         // FP32 HR table kept in shared memory
  // threads per block of the persistent kernel (bounds the register budget)
  static constexpr int THREADS = N <= 45 ? 512 : (N <= 66 ? 384 : 192);
  // threads per block of the phased solve kernel (no FP32 table, split assembly)
  // (its register budget is 65536 / SOLVE_THREADS; CSD_SOLVE_THREADS45
  // overrides it for N <= 45)
#ifdef CSD_SOLVE_THREADS45
  static constexpr int SOLVE_THREADS = N <= 45 ? CSD_SOLVE_THREADS45 : THREADS;
#else
  static constexpr int SOLVE_THREADS = N <= 45 ? 640 : THREADS;
#endif
};

// Exact power of two 2^k as a float (k clamped to the normal range).
__host__ __device__ __forceinline__ float pow2f(int k) {
  k = k < -126 ? -126 : (k > 127 ? 127 : k);
  union {
    unsigned u;
    float f;
  } x;
  x.u = (unsigned)(k + 127) << 23;
  return x.f;
}

// Exponent that brings the largest of n values (>= 0) into [2^14, 2^15):
// scaling by 2^-e keeps FP16 hi halves below 65504 and lo halves of the
// large entries normal, at any scale of the caller's data (the reference's
// FOD is scale-covariant: F(a S, b r) = (a / b) F(S, r)).  0 for all-zero data.
__device__ __forceinline__ int fp16_split_exponent(float maxabs) {
  if (!(maxabs > 0.f) || !isfinite(maxabs)) return 0;
  return ((__float_as_int(maxabs) >> 23) & 0xFF) - 127 - 14;
}

// Everything a voxel of one image needs, by device pointer.
struct Scheme {
  const float* H32;       // [nhr][HS] HR_trans, fp32, zero padded
  const __half* H16;      // [2][nhr+1][HS16] HR_trans / hscale, hi then lo, fp16, row nhr = 0
  const double* H64;      // [nhr][nsh] HR_trans, fp64 (FP64 fallback)
  const float* MtMp;      // packed-padded lower Mt_M, fp32
  const double* MtM64;    // [nsh][nsh] full Mt_M, fp64 (refinement residual)
  const float* rconvT;    // [ndw][ninit] rconv^T, fp32
  const float* M32;       // [ndw][nsh] M, fp32
  const int* dwis;        // [ndw]
  int ndw, ninit, niter;
  float threshold;
  float hscale;           // power of two: the FP16 tables hold HR_trans / hscale
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
  int fast_cycles;               // jump exactly periodic two-cycles to their last call
  float cond_thr;
  long long total;
  unsigned long long* queue;     // work counter, zeroed before launch
  double* fp64_scratch;          // [gridDim.x * warps][WSZ] doubles
  VolumeDesc vol[kMaxVolumesPerLaunch];
};

// Bytes of the constraint tables a block keeps in shared memory.
template <int N>
__host__ __device__ constexpr int htab_bytes_32(int nhr, bool use32 = true) {
  return (Dims<N>::KEEP32 && use32) ? ((nhr * Dims<N>::HS * 4 + 15) / 16) * 16 : 0;
}
template <int N>
__host__ __device__ constexpr int htab_bytes(int nhr, bool use32 = true) {
  return htab_bytes_32<N>(nhr, use32) + 2 * (nhr + 1) * Dims<N>::HS16 * 2;
}

// Shared-memory view of the constraint tables.
template <int N>
struct HTab {
  const float* h32;   // [nhr][HS] (KEEP32 only)
  const __half* hh;   // [nhr+1][HS16]
  const __half* hl;   // [nhr+1][HS16]
  int nhr;
  bool use32;         // read FP32 values from h32 (else re-sum the FP16 pair)
  float hs;           // power of two the FP16 pair is scaled down by

  // FP32 values of row d, columns 4j..4j+3
  __device__ __forceinline__ float4 quad(int d, int j) const {
    if (Dims<N>::KEEP32 && use32) {
      return reinterpret_cast<const float4*>(h32 + d * Dims<N>::HS)[j];
    } else {
      const uint2 a = *reinterpret_cast<const uint2*>(hh + d * Dims<N>::HS16 + 4 * j);
      const uint2 b = *reinterpret_cast<const uint2*>(hl + d * Dims<N>::HS16 + 4 * j);
      const float2 a0 = __half22float2(*reinterpret_cast<const __half2*>(&a.x));
      const float2 a1 = __half22float2(*reinterpret_cast<const __half2*>(&a.y));
      const float2 b0 = __half22float2(*reinterpret_cast<const __half2*>(&b.x));
      const float2 b1 = __half22float2(*reinterpret_cast<const __half2*>(&b.y));
      return make_float4((a0.x + b0.x) * hs, (a0.y + b0.y) * hs, (a1.x + b1.x) * hs, (a1.y + b1.y) * hs);
    }
  }
  __device__ __forceinline__ float val(int d, int i) const {
    if (Dims<N>::KEEP32 && use32) {
      return h32[d * Dims<N>::HS + i];
    } else {
      return (__half2float(hh[d * Dims<N>::HS16 + i]) + __half2float(hl[d * Dims<N>::HS16 + i])) * hs;
    }
  }
};

// Copy a scheme's constraint tables into shared memory (whole block).
template <int N>
__device__ HTab<N> load_htab(unsigned char* smem, const Scheme& sc, int nhr, bool use32 = true) {
  HTab<N> t;
  t.nhr = nhr;
  t.use32 = Dims<N>::KEEP32 && use32;
  t.hs = sc.hscale;
  const int b32 = htab_bytes_32<N>(nhr, use32);
  t.h32 = reinterpret_cast<const float*>(smem);
  if (t.use32) {
    const float4* src = reinterpret_cast<const float4*>(sc.H32);
    float4* dst = reinterpret_cast<float4*>(smem);
    for (int i = threadIdx.x; i < nhr * Dims<N>::HS / 4; i += blockDim.x) dst[i] = __ldg(src + i);
  }
  const int n16 = 2 * (nhr + 1) * Dims<N>::HS16;  // halves, a multiple of 8
  const uint4* src = reinterpret_cast<const uint4*>(sc.H16);
  uint4* dst = reinterpret_cast<uint4*>(smem + b32);
  for (int i = threadIdx.x; i < n16 / 8; i += blockDim.x) dst[i] = __ldg(src + i);
  t.hh = reinterpret_cast<const __half*>(smem + b32);
  t.hl = t.hh + (nhr + 1) * Dims<N>::HS16;
  return t;
}

// Per-warp shared-memory workspace (carved from dynamic shared memory).
template <int N>
__host__ __device__ constexpr int wbuf_floats() {
  // packed W plus one appended row (the right-hand side during factorisation)
  return packoff(N + 1) > kMaxDW ? packoff(N + 1) : kMaxDW;
}

template <int N>
struct WarpWS {
  float* W;        // packed W / L (also holds S during set)
  float* F;        // [HS] current F (fp32)
  float* rdiag;    // [N] 1 / L_ii
  double* b;       // [N] M^T S (fp64)
  uint16_t* neg;   // [kMaxHR] negative-set index list
  uint32_t* old;   // [kMaxWords] negative set of the last solve (bitmask)
  uint32_t* old2;  // [kMaxWords] negative set of the solve before
};

template <int N>
__host__ __device__ constexpr int rdiag_bytes() {
  return ((N * 4 + 15) / 16) * 16;
}

template <int N>
__host__ __device__ constexpr int warp_ws_bytes() {
  return wbuf_floats<N>() * 4 + Dims<N>::HS * 4 + rdiag_bytes<N>() + ((N * 8 + 15) / 16) * 16 + kMaxHR * 2 +
         2 * kMaxWords * 4;
}

template <int N>
__device__ __forceinline__ WarpWS<N> carve_ws(unsigned char* base) {
  WarpWS<N> w;
  w.W = reinterpret_cast<float*>(base);
  w.F = w.W + wbuf_floats<N>();
  w.rdiag = w.F + Dims<N>::HS;
  w.b = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(w.rdiag) + rdiag_bytes<N>());
  w.neg = reinterpret_cast<uint16_t*>(reinterpret_cast<unsigned char*>(w.b) + ((N * 8 + 15) / 16) * 16);
  w.old = reinterpret_cast<uint32_t*>(w.neg + kMaxHR);
  w.old2 = w.old + kMaxWords;
  return w;
}

__device__ __forceinline__ double shfl_d(double v, int src) {
  return __shfl_sync(0xffffffffu, v, src);
}

// ---------------------------------------------------------------------------
// set(): load + clamp the voxel's DW samples (dwi2fod.cpp:156-173), then
// F = [rconv S; 0] and b = M^T S (csd.h:237-243) in FP32 (b kept as double
// for the refinement residual).  Returns 0 = ok, 1 = masked out, 3 =
// non-finite sample.
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
  const int nd4 = sc.ndw & ~3;
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int c = lane + 32 * q;
    float f0 = 0.f, f1 = 0.f, b0 = 0.f, b1 = 0.f;
    if (c < N) {
      const bool hasf = c < sc.ninit;
      const float* rc = sc.rconvT + c;
      const float* mc = sc.M32 + c;
      int t = 0;
      for (; t < nd4; t += 4) {
        const float4 s4 = *reinterpret_cast<const float4*>(S + t);
        if (hasf) {
          f0 = fmaf(__ldg(rc + (long long)t * sc.ninit), s4.x, f0);
          f1 = fmaf(__ldg(rc + (long long)(t + 1) * sc.ninit), s4.y, f1);
          f0 = fmaf(__ldg(rc + (long long)(t + 2) * sc.ninit), s4.z, f0);
          f1 = fmaf(__ldg(rc + (long long)(t + 3) * sc.ninit), s4.w, f1);
        }
        b0 = fmaf(__ldg(mc + (long long)t * N), s4.x, b0);
        b1 = fmaf(__ldg(mc + (long long)(t + 1) * N), s4.y, b1);
        b0 = fmaf(__ldg(mc + (long long)(t + 2) * N), s4.z, b0);
        b1 = fmaf(__ldg(mc + (long long)(t + 3) * N), s4.w, b1);
      }
      for (; t < sc.ndw; ++t) {
        if (hasf) f0 = fmaf(__ldg(rc + (long long)t * sc.ninit), S[t], f0);
        b0 = fmaf(__ldg(mc + (long long)t * N), S[t], b0);
      }
      w.b[c] = (double)(b0 + b1);
    }
    if (c < Dims<N>::HS) w.F[c] = (c < N) ? (f0 + f1) : 0.f;
  }
  for (int c = lane + 32 * Dims<N>::CQ; c < Dims<N>::HS; c += 32) w.F[c] = 0.f;
  __syncwarp();
  return 0;
}

// ---------------------------------------------------------------------------
// Projection onto the constraint directions and the negative-set bitmask
// (csd.h:246-250).  Lane l evaluates directions l, l+32, ...; F is read as
// broadcast float4s.
template <int N>
__device__ __forceinline__ void project_mask(const HTab<N>& H, int nw, float thr, const WarpWS<N>& w, int lane,
                                             uint32_t* bits) {
  const int nhr = H.nhr;
  float acc[kMaxWords];
#pragma unroll
  for (int p = 0; p < kMaxWords; ++p) acc[p] = 0.f;
#pragma unroll 4
  for (int j = 0; j < Dims<N>::NQ; ++j) {
    const float4 f4 = reinterpret_cast<const float4*>(w.F)[j];
#pragma unroll
    for (int p = 0; p < kMaxWords; ++p) {
      if (p < nw) {
        const int d = lane + 32 * p;
        if (d < nhr) {
          const float4 h4 = H.quad(d, j);
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
// Tensor-core rank-k assembly: W = Mt_M + G^T G, G = HR_trans rows in neg
// (csd.h:255-262).  As a GEMM, A = G^T (N x k) and B = G (k x N); both
// fragments of m16n8k16 come from ldmatrix.trans on 8x8 blocks of G, whose
// rows are the table rows neg[q] -- each lane hands ldmatrix one row
// address, so the gather costs nothing.  Only the lower triangle's tiles
// are computed: row block ib (16 rows) x column block jb (8 columns),
// jb <= 2 ib + 1.  Row blocks [IB0, IB1) are accumulated in this pass.

__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const __half* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void ldsm_x4_trans(uint32_t (&r)[4], const __half* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void mma_f16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int N, int IB0, int IB1>
__device__ __forceinline__ void assemble_pass(const HTab<N>& H, const float* MtMp, int k, const WarpWS<N>& w,
                                              int lane) {
  using D = Dims<N>;
  constexpr int NJ = 2 * IB1 < D::NJB ? 2 * IB1 : D::NJB;  // column blocks touched
  float acc[IB1 - IB0][NJ][4];
#pragma unroll
  for (int a = 0; a < IB1 - IB0; ++a)
#pragma unroll
    for (int c = 0; c < NJ; ++c)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[a][c][e] = 0.f;
  const int qsel = (lane & 7) + 8 * (lane >> 4);
  const int csel = 8 * ((lane >> 3) & 1);
#pragma unroll 1
  for (int k0 = 0; k0 < k; k0 += 16) {
    const int q = k0 + qsel;
    const int d = q < k ? (int)w.neg[q] : H.nhr;  // row nhr of the tables is zero
    const __half* ph = H.hh + d * D::HS16 + csel;
    const __half* pl = H.hl + d * D::HS16 + csel;
    uint32_t ah[IB1][4], al[IB1][4];
#pragma unroll
    for (int b = 0; b < IB1; ++b) {
      ldsm_x4_trans(ah[b], ph + 16 * b);
      ldsm_x4_trans(al[b], pl + 16 * b);
    }
#pragma unroll
    for (int ib = IB0; ib < IB1; ++ib) {
#pragma unroll
      for (int jb = 0; jb < NJ; ++jb) {
        if (jb <= 2 * ib + 1) {
          const int bb = jb >> 1, hs = jb & 1;
          mma_f16(acc[ib - IB0][jb], ah[ib], ah[bb][hs], ah[bb][2 + hs]);
          mma_f16(acc[ib - IB0][jb], ah[ib], al[bb][hs], al[bb][2 + hs]);
          mma_f16(acc[ib - IB0][jb], al[ib], ah[bb][hs], ah[bb][2 + hs]);
        }
      }
    }
  }
  const int gid = lane >> 2, tig = lane & 3;
  const float ws = H.hs * H.hs;  // exact: the tables are HR_trans / hs
#pragma unroll
  for (int ib = IB0; ib < IB1; ++ib) {
#pragma unroll
    for (int jb = 0; jb < NJ; ++jb) {
      if (jb <= 2 * ib + 1) {
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          const int i = 16 * ib + gid + 8 * r;
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int j = 8 * jb + 2 * tig + c;
            if (i < N && j <= i) {
              const int o = packoff(i) + j;
              w.W[o] = __ldg(MtMp + o) + acc[ib - IB0][jb][2 * r + c] * ws;
            }
          }
        }
      }
    }
  }
}

template <int N, bool SPLIT = false>
__device__ void assemble(const HTab<N>& H, const float* MtMp, int k, const WarpWS<N>& w, int lane) {
  constexpr int R = Dims<N>::NRB;
  if constexpr (SPLIT && R == 3) {
    // one 16-row block per pass: fewer live accumulators for high occupancy
    assemble_pass<N, 0, 1>(H, MtMp, k, w, lane);
    assemble_pass<N, 1, 2>(H, MtMp, k, w, lane);
    assemble_pass<N, 2, 3>(H, MtMp, k, w, lane);
  } else if constexpr (R <= 3) {
    assemble_pass<N, 0, R>(H, MtMp, k, w, lane);
  } else if constexpr (R <= 5) {
    assemble_pass<N, 0, 3>(H, MtMp, k, w, lane);
    assemble_pass<N, 3, R>(H, MtMp, k, w, lane);
  } else {
    assemble_pass<N, 0, 3>(H, MtMp, k, w, lane);
    assemble_pass<N, 3, 5>(H, MtMp, k, w, lane);
    assemble_pass<N, 5, R>(H, MtMp, k, w, lane);
  }
  __syncwarp();
}

// ---------------------------------------------------------------------------
// In-place left-looking Cholesky of the packed-padded lower matrix A (shared
// or global memory), FP64 version for the fallback.  Lane l computes rows
// j+l, j+l+32, ... of column j.  Returns false if a pivot is not positive.
template <int N, typename T>
__device__ bool cholesky_packed(T* A, int lane) {
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
    if (!(djj > (T)0)) return false;
    const T d = sqrt(djj);
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

// FP32 version, blocked by 4 columns: for column block [j0, j0+4) every
// active row i >= j0 (lane i - j0 + 32 q) forms s_c = A[i][j0+c] -
// L[i][0:j0] . L[j0+c][0:j0] with one float4 of its own row against four
// broadcast float4s per step; the 4x4 diagonal block is then factored by
// every lane from shuffled values, and the rows below divide through it.
// Stores 1/L_jj in rdiag; dmin/dmax receive the range of diag(L).
template <int N>
__device__ bool cholesky_packed_f32(float* A, float* rdiag, int lane, float& dmin, float& dmax) {
  dmin = 3.0e38f;
  dmax = 0.f;
  constexpr int NB = (N + 3) / 4;
CSD_CHOL_CB_PRAGMA
  for (int cb = 0; cb < NB; ++cb) {
    const int j0 = 4 * cb;
    const float* Lj0 = A + packoff(j0);
    const float* Lj1 = A + packoff(j0 + 1);
    const float* Lj2 = A + packoff(j0 + 2);
    const float* Lj3 = A + packoff(j0 + 3);
    float s[Dims<N>::CQ][4];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j0 + lane + 32 * q;
#pragma unroll
      for (int c = 0; c < 4; ++c) s[q][c] = 0.f;
      if (i <= N) {  // row N is the appended right-hand side
        const float* Li = A + packoff(i);
        const float4 w4 = *reinterpret_cast<const float4*>(Li + j0);
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f, b0 = 0.f, b1 = 0.f, b2 = 0.f, b3 = 0.f;
CSD_CHOL_KK_PRAGMA
        for (int kk = 0; kk < j0; kk += 4) {
          const float4 x = *reinterpret_cast<const float4*>(Li + kk);
          const float4 y0 = *reinterpret_cast<const float4*>(Lj0 + kk);
          const float4 y1 = *reinterpret_cast<const float4*>(Lj1 + kk);
          const float4 y2 = *reinterpret_cast<const float4*>(Lj2 + kk);
          const float4 y3 = *reinterpret_cast<const float4*>(Lj3 + kk);
          a0 = fmaf(x.x, y0.x, a0); b0 = fmaf(x.y, y0.y, b0); a0 = fmaf(x.z, y0.z, a0); b0 = fmaf(x.w, y0.w, b0);
          a1 = fmaf(x.x, y1.x, a1); b1 = fmaf(x.y, y1.y, b1); a1 = fmaf(x.z, y1.z, a1); b1 = fmaf(x.w, y1.w, b1);
          a2 = fmaf(x.x, y2.x, a2); b2 = fmaf(x.y, y2.y, b2); a2 = fmaf(x.z, y2.z, a2); b2 = fmaf(x.w, y2.w, b2);
          a3 = fmaf(x.x, y3.x, a3); b3 = fmaf(x.y, y3.y, b3); a3 = fmaf(x.z, y3.z, a3); b3 = fmaf(x.w, y3.w, b3);
        }
        s[q][0] = w4.x - (a0 + b0);
        s[q][1] = w4.y - (a1 + b1);
        s[q][2] = w4.z - (a2 + b2);
        s[q][3] = w4.w - (a3 + b3);
      }
    }
    // the diagonal block rows j0..j0+3 sit in lanes 0..3 of slot 0
    float d[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
      for (int c = 0; c <= t; ++c) d[t][c] = __shfl_sync(0xffffffffu, s[0][c], t);
    // rows t < nb of the block are matrix rows; row t == nb, if it is N, is
    // the right-hand side (off-diagonal part only); rows beyond are unused
    const int nb = N - j0 < 4 ? N - j0 : 4;
    float L[4][4], rd[4];
    bool ok = true;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
#pragma unroll
      for (int c = 0; c < t; ++c) {
        float v = d[t][c];
#pragma unroll
        for (int e = 0; e < c; ++e) v = fmaf(-L[t][e], L[c][e], v);
        L[t][c] = (t <= nb && c < nb) ? v * rd[c] : 0.f;
      }
      float v = d[t][t];
#pragma unroll
      for (int e = 0; e < t; ++e) v = fmaf(-L[t][e], L[t][e], v);
      if (t >= nb) v = 1.f;  // the right-hand-side row and rows past it: identity
      ok = ok && (v > 0.f) && isfinite(v);
      const float dd = sqrtf(v);
      L[t][t] = dd;
      rd[t] = 1.0f / dd;
      if (t < nb) {
        dmin = fminf(dmin, dd);
        dmax = fmaxf(dmax, dd);
      }
    }
    if (!ok) return false;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = j0 + lane + 32 * q;
      if (i <= N) {
        float o[4];
        if (q == 0 && lane < 4) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float v = 0.f;
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (t == lane && c <= t) v = L[t][c];
            o[c] = v;
          }
        } else {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float v = s[q][c];
#pragma unroll
            for (int e = 0; e < c; ++e) v = fmaf(-o[e], L[c][e], v);
            o[c] = v * rd[c];
          }
        }
        *reinterpret_cast<float4*>(A + packoff(i) + j0) = make_float4(o[0], o[1], o[2], o[3]);
      }
    }
    if (lane < 4) rdiag[j0 + lane] = lane == 0 ? rd[0] : lane == 1 ? rd[1] : lane == 2 ? rd[2] : rd[3];
    __syncwarp();
  }
  return true;
}

// x := L^-T L^-1 x with x distributed as x[q] = element lane + 32 q, blocked
// by 4: each block's four unknowns are gathered by shuffles, solved against
// the 4x4 diagonal block, and pushed into the remaining rows with one float4
// (forward) or four scalars (backward) of L per row.
template <int N>
__device__ __forceinline__ void chol_subst_f32(const float* L, const float* rdiag, float* x, int lane) {
  constexpr int NB = (N + 3) / 4;
#pragma unroll 1
  for (int cb = 0; cb < NB; ++cb) {
    const int j0 = 4 * cb;
    float y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = j0 + c;
      float xv = 0.f;
#pragma unroll
      for (int q = 0; q < Dims<N>::CQ; ++q)
        if (q == (r >> 5)) xv = x[q];
      y[c] = __shfl_sync(0xffffffffu, xv, r & 31);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      if (j0 + c < N) {
        const float* Lc = L + packoff(j0 + c) + j0;
        float v = y[c];
#pragma unroll
        for (int e = 0; e < c; ++e) v = fmaf(-Lc[e], y[e], v);
        y[c] = v * rdiag[j0 + c];
      } else {
        y[c] = 0.f;
      }
    }
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i >= j0 + 4 && i < N) {
        const float4 l4 = *reinterpret_cast<const float4*>(L + packoff(i) + j0);
        x[q] = fmaf(-l4.x, y[0], x[q]);
        x[q] = fmaf(-l4.y, y[1], x[q]);
        x[q] = fmaf(-l4.z, y[2], x[q]);
        x[q] = fmaf(-l4.w, y[3], x[q]);
      } else if (i >= j0 && i < j0 + 4 && i < N) {
        x[q] = (i == j0) ? y[0] : (i == j0 + 1) ? y[1] : (i == j0 + 2) ? y[2] : y[3];
      }
    }
  }
#pragma unroll 1
  for (int cb = NB - 1; cb >= 0; --cb) {
    const int j0 = 4 * cb;
    float y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = j0 + c;
      float xv = 0.f;
#pragma unroll
      for (int q = 0; q < Dims<N>::CQ; ++q)
        if (q == (r >> 5)) xv = x[q];
      y[c] = __shfl_sync(0xffffffffu, xv, r & 31);
    }
#pragma unroll
    for (int c = 3; c >= 0; --c) {
      if (j0 + c < N) {
        float v = y[c];
#pragma unroll
        for (int e = c + 1; e < 4; ++e)
          if (j0 + e < N) v = fmaf(-L[packoff(j0 + e) + j0 + c], y[e], v);
        y[c] = v * rdiag[j0 + c];
      } else {
        y[c] = 0.f;
      }
    }
    const float* L0 = L + packoff(j0);
    const float* L1 = L + packoff(j0 + 1);
    const float* L2 = L + packoff(j0 + 2);
    const float* L3 = L + packoff(j0 + 3);
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < j0) {
        float v = x[q];
        v = fmaf(-L0[i], y[0], v);
        if (j0 + 1 < N) v = fmaf(-L1[i], y[1], v);
        if (j0 + 2 < N) v = fmaf(-L2[i], y[2], v);
        if (j0 + 3 < N) v = fmaf(-L3[i], y[3], v);
        x[q] = v;
      } else if (i < j0 + 4 && i < N) {
        x[q] = (i == j0) ? y[0] : (i == j0 + 1) ? y[1] : (i == j0 + 2) ? y[2] : y[3];
      }
    }
  }
}

// x := L^-T x (the backward half of chol_subst_f32), x distributed as above.
template <int N>
__device__ __forceinline__ void chol_back_f32(const float* L, const float* rdiag, float* x, int lane) {
  constexpr int NB = (N + 3) / 4;
CSD_BACK_CB_PRAGMA
  for (int cb = NB - 1; cb >= 0; --cb) {
    const int j0 = 4 * cb;
    float y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = j0 + c;
      float xv = 0.f;
#pragma unroll
      for (int q = 0; q < Dims<N>::CQ; ++q)
        if (q == (r >> 5)) xv = x[q];
      y[c] = __shfl_sync(0xffffffffu, xv, r & 31);
    }
#pragma unroll
    for (int c = 3; c >= 0; --c) {
      if (j0 + c < N) {
        float v = y[c];
#pragma unroll
        for (int e = c + 1; e < 4; ++e)
          if (j0 + e < N) v = fmaf(-L[packoff(j0 + e) + j0 + c], y[e], v);
        y[c] = v * rdiag[j0 + c];
      } else {
        y[c] = 0.f;
      }
    }
    const float* L0 = L + packoff(j0);
    const float* L1 = L + packoff(j0 + 1);
    const float* L2 = L + packoff(j0 + 2);
    const float* L3 = L + packoff(j0 + 3);
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < j0) {
        float v = x[q];
        v = fmaf(-L0[i], y[0], v);
        if (j0 + 1 < N) v = fmaf(-L1[i], y[1], v);
        if (j0 + 2 < N) v = fmaf(-L2[i], y[2], v);
        if (j0 + 3 < N) v = fmaf(-L3[i], y[3], v);
        x[q] = v;
      } else if (i < j0 + 4 && i < N) {
        x[q] = (i == j0) ? y[0] : (i == j0 + 1) ? y[1] : (i == j0 + 2) ? y[2] : y[3];
      }
    }
  }
}

// ---- grouped variants: G lanes per system, 32 / G systems per warp.  Each
// group runs the exact operation sequence of cholesky_packed_f32 /
// chol_back_f32 on its own matrix (sublane s in place of the lane, G in
// place of 32, shuffles of width G), so the results are bit-identical to
// the warp-per-system versions while one warp instruction serves 32 / G
// systems and fewer lanes idle on the short rows of late column blocks.
template <int N, int G>
struct GroupDims {
  static constexpr int V = 32 / G;               // systems per warp
  static constexpr int CQG = (N + 1 + G - 1) / G;  // row slots per lane (rows 0..N)
};

// Factorisation of the group's packed matrix A (rows 0..N, row N the
// right-hand side).  Never returns early: the shuffles need every lane of
// the warp, so a failed pivot only clears the returned flag (group-uniform).
template <int N, int G>
__device__ bool cholesky_group_f32(float* A, float* rdiag, int s, float& dmin, float& dmax) {
  constexpr int CQG = GroupDims<N, G>::CQG;
  dmin = 3.0e38f;
  dmax = 0.f;
  bool okall = true;
  constexpr int NB = (N + 3) / 4;
CSD_CHOL_CB_PRAGMA
  for (int cb = 0; cb < NB; ++cb) {
    const int j0 = 4 * cb;
    const float* Lj0 = A + packoff(j0);
    const float* Lj1 = A + packoff(j0 + 1);
    const float* Lj2 = A + packoff(j0 + 2);
    const float* Lj3 = A + packoff(j0 + 3);
    // every row slot of this lane in one pass over k: the four pivot-row
    // quads are loaded once per step and shared by the slots, whose chains
    // are independent (the same fmaf sequence per element as the warp form)
    const float* Li[CQG];
    bool act[CQG];
    float acc[CQG][8];
#pragma unroll
    for (int q = 0; q < CQG; ++q) {
      const int i = j0 + s + G * q;
      act[q] = i <= N;
      Li[q] = A + packoff(act[q] ? i : j0);
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[q][c] = 0.f;
    }
    CSD_CHOL_KK_PRAGMA
    for (int kk = 0; kk < j0; kk += 4) {
      const float4 y0 = *reinterpret_cast<const float4*>(Lj0 + kk);
      const float4 y1 = *reinterpret_cast<const float4*>(Lj1 + kk);
      const float4 y2 = *reinterpret_cast<const float4*>(Lj2 + kk);
      const float4 y3 = *reinterpret_cast<const float4*>(Lj3 + kk);
#pragma unroll
      for (int q = 0; q < CQG; ++q) {
        if (act[q]) {
          const float4 x = *reinterpret_cast<const float4*>(Li[q] + kk);
          float* a = acc[q];
          a[0] = fmaf(x.x, y0.x, a[0]); a[4] = fmaf(x.y, y0.y, a[4]); a[0] = fmaf(x.z, y0.z, a[0]); a[4] = fmaf(x.w, y0.w, a[4]);
          a[1] = fmaf(x.x, y1.x, a[1]); a[5] = fmaf(x.y, y1.y, a[5]); a[1] = fmaf(x.z, y1.z, a[1]); a[5] = fmaf(x.w, y1.w, a[5]);
          a[2] = fmaf(x.x, y2.x, a[2]); a[6] = fmaf(x.y, y2.y, a[6]); a[2] = fmaf(x.z, y2.z, a[2]); a[6] = fmaf(x.w, y2.w, a[6]);
          a[3] = fmaf(x.x, y3.x, a[3]); a[7] = fmaf(x.y, y3.y, a[7]); a[3] = fmaf(x.z, y3.z, a[3]); a[7] = fmaf(x.w, y3.w, a[7]);
        }
      }
    }
    float sv[CQG][4];
#pragma unroll
    for (int q = 0; q < CQG; ++q) {
#pragma unroll
      for (int c = 0; c < 4; ++c) sv[q][c] = 0.f;
      if (act[q]) {
        const float4 w4 = *reinterpret_cast<const float4*>(Li[q] + j0);
        sv[q][0] = w4.x - (acc[q][0] + acc[q][4]);
        sv[q][1] = w4.y - (acc[q][1] + acc[q][5]);
        sv[q][2] = w4.z - (acc[q][2] + acc[q][6]);
        sv[q][3] = w4.w - (acc[q][3] + acc[q][7]);
      }
    }
    // the diagonal block rows j0..j0+3 sit in sublanes 0..3 of slot 0
    float d[4][4];
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
      for (int c = 0; c <= t; ++c) d[t][c] = __shfl_sync(0xffffffffu, sv[0][c], t, G);
    const int nb = N - j0 < 4 ? N - j0 : 4;
    float L[4][4], rd[4];
    bool ok = true;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
#pragma unroll
      for (int c = 0; c < t; ++c) {
        float v = d[t][c];
#pragma unroll
        for (int e = 0; e < c; ++e) v = fmaf(-L[t][e], L[c][e], v);
        L[t][c] = (t <= nb && c < nb) ? v * rd[c] : 0.f;
      }
      float v = d[t][t];
#pragma unroll
      for (int e = 0; e < t; ++e) v = fmaf(-L[t][e], L[t][e], v);
      if (t >= nb) v = 1.f;
      ok = ok && (v > 0.f) && isfinite(v);
      const float dd = sqrtf(v);
      L[t][t] = dd;
      rd[t] = 1.0f / dd;
      if (t < nb) {
        dmin = fminf(dmin, dd);
        dmax = fmaxf(dmax, dd);
      }
    }
    okall = okall && ok;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < CQG; ++q) {
      const int i = j0 + s + G * q;
      if (i <= N) {
        float o[4];
        if (q == 0 && s < 4) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float v = 0.f;
#pragma unroll
            for (int t = 0; t < 4; ++t)
              if (t == s && c <= t) v = L[t][c];
            o[c] = v;
          }
        } else {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float v = sv[q][c];
#pragma unroll
            for (int e = 0; e < c; ++e) v = fmaf(-o[e], L[c][e], v);
            o[c] = v * rd[c];
          }
        }
        *reinterpret_cast<float4*>(A + packoff(i) + j0) = make_float4(o[0], o[1], o[2], o[3]);
      }
    }
    if (s < 4) rdiag[j0 + s] = s == 0 ? rd[0] : s == 1 ? rd[1] : s == 2 ? rd[2] : rd[3];
    __syncwarp();
  }
  return okall;
}

// x := L^-T x for the group's factor, x distributed as x[q] = element s + G q.
template <int N, int G>
__device__ __forceinline__ void chol_back_group_f32(const float* L, const float* rdiag, float* x, int s) {
  constexpr int CQG = GroupDims<N, G>::CQG;
  constexpr int NB = (N + 3) / 4;
CSD_BACK_CB_PRAGMA
  for (int cb = NB - 1; cb >= 0; --cb) {
    const int j0 = 4 * cb;
    float y[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int r = j0 + c;
      float xv = 0.f;
#pragma unroll
      for (int q = 0; q < CQG; ++q)
        if (q == r / G) xv = x[q];
      y[c] = __shfl_sync(0xffffffffu, xv, r % G, G);
    }
#pragma unroll
    for (int c = 3; c >= 0; --c) {
      if (j0 + c < N) {
        float v = y[c];
#pragma unroll
        for (int e = c + 1; e < 4; ++e)
          if (j0 + e < N) v = fmaf(-L[packoff(j0 + e) + j0 + c], y[e], v);
        y[c] = v * rdiag[j0 + c];
      } else {
        y[c] = 0.f;
      }
    }
    const float* L0 = L + packoff(j0);
    const float* L1 = L + packoff(j0 + 1);
    const float* L2 = L + packoff(j0 + 2);
    const float* L3 = L + packoff(j0 + 3);
#pragma unroll
    for (int q = 0; q < CQG; ++q) {
      const int i = s + G * q;
      if (i < j0) {
        float v = x[q];
        v = fmaf(-L0[i], y[0], v);
        if (j0 + 1 < N) v = fmaf(-L1[i], y[1], v);
        if (j0 + 2 < N) v = fmaf(-L2[i], y[2], v);
        if (j0 + 3 < N) v = fmaf(-L3[i], y[3], v);
        x[q] = v;
      } else if (i < j0 + 4 && i < N) {
        x[q] = (i == j0) ? y[0] : (i == j0 + 1) ? y[1] : (i == j0 + 2) ? y[2] : y[3];
      }
    }
  }
}

// Per-warp workspace of the grouped solve: V slots, each [packed W + the
// right-hand-side row][F][1/L_ii][b (fp64)], then one negative-set list
// shared by the slots (the assembly uses it one slot at a time).  The slot
// stride is padded to 128/V bytes past a multiple of 128 so the groups'
// scalar accesses at equal offsets fall in different banks.
template <int N, int V>
struct GroupWSLayout {
  static constexpr int W_BYTES = ((packoff(N + 1) * 4 + 15) / 16) * 16;
  static constexpr int F_BYTES = Dims<N>::HS * 4;
  static constexpr int B_BYTES = ((N * 8 + 15) / 16) * 16;
  static constexpr int RAW = W_BYTES + F_BYTES + rdiag_bytes<N>() + B_BYTES;
  static constexpr int PAD = 128 / V;
  static constexpr int SLOT = ((RAW - PAD + 127) / 128) * 128 + PAD;
  static constexpr int WARP = V * SLOT + ((kMaxHR * 2 + 15) / 16) * 16;
};

template <int N, int V>
__device__ __forceinline__ WarpWS<N> group_slot_ws(unsigned char* base, int g) {
  using Lw = GroupWSLayout<N, V>;
  WarpWS<N> w;
  unsigned char* p = base + g * Lw::SLOT;
  w.W = reinterpret_cast<float*>(p);
  w.F = reinterpret_cast<float*>(p + Lw::W_BYTES);
  w.rdiag = reinterpret_cast<float*>(p + Lw::W_BYTES + Lw::F_BYTES);
  w.b = reinterpret_cast<double*>(p + Lw::W_BYTES + Lw::F_BYTES + rdiag_bytes<N>());
  w.neg = reinterpret_cast<uint16_t*>(base + V * Lw::SLOT);
  w.old = nullptr;
  w.old2 = nullptr;
  return w;
}

// FP64 version (fallback path, L in FP64 global scratch).
template <int N>
__device__ __forceinline__ void chol_subst_f64(const double* L, double* x, int lane) {
#pragma unroll 1
  for (int kk = 0; kk < N; ++kk) {
    const int src = kk & 31, slot = kk >> 5;
    double xv = 0.0;
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q)
      if (q == slot) xv = x[q];
    const double xk = shfl_d(xv, src) / L[packoff(kk) + kk];
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i > kk && i < N) x[q] -= L[packoff(i) + kk] * xk;
      if (i == kk) x[q] = xk;
    }
  }
#pragma unroll 1
  for (int kk = N - 1; kk >= 0; --kk) {
    const int src = kk & 31, slot = kk >> 5;
    double xv = 0.0;
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q)
      if (q == slot) xv = x[q];
    const double xk = shfl_d(xv, src) / L[packoff(kk) + kk];
    const double* Lk = L + packoff(kk);
#pragma unroll
    for (int q = 0; q < Dims<N>::CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < kk) x[q] -= Lk[i] * xk;
      if (i == kk) x[q] = xk;
    }
  }
}

// r = b - (Mt_M F + sum_{d in neg} h_d (h_d . F)), accumulated in FP64 with
// the FP32 operators.  F is read from w.F.
template <int N>
__device__ void residual_fp64(const Scheme& sc, const HTab<N>& H, int k, const WarpWS<N>& w, int lane,
                              double* r) {
  double u[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) u[q] = 0.0;
  for (int q0 = 0; q0 < k; q0 += 32) {
    const int qq = q0 + lane;
    double t = 0.0;
    if (qq < k) {
      const int d = (int)w.neg[qq];
      const float4* f = reinterpret_cast<const float4*>(w.F);
#pragma unroll 4
      for (int j = 0; j < Dims<N>::NQ; ++j) {
        const float4 a = H.quad(d, j), c = f[j];
        t = fma((double)a.x, (double)c.x, t);
        t = fma((double)a.y, (double)c.y, t);
        t = fma((double)a.z, (double)c.z, t);
        t = fma((double)a.w, (double)c.w, t);
      }
    }
    const int cnt = min(32, k - q0);
    for (int s = 0; s < cnt; ++s) {
      const double ts = shfl_d(t, s);
      const int d = (int)w.neg[q0 + s];
#pragma unroll
      for (int q = 0; q < Dims<N>::CQ; ++q) {
        const int i = lane + 32 * q;
        if (i < N) u[q] = fma(ts, (double)H.val(d, i), u[q]);
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

// One refinement step of the current solution in w.F, with the FP32 factor
// still in w.W / w.rdiag and the set in w.neg[0..k).
template <int N>
__device__ void refine_step(const Scheme& sc, const HTab<N>& H, int k, const WarpWS<N>& w, int lane) {
  double r[Dims<N>::CQ];
  residual_fp64<N>(sc, H, k, w, lane, r);
  float d[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) d[q] = (float)r[q];
  chol_subst_f32<N>(w.W, w.rdiag, d, lane);
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    if (i < N) w.F[i] += d[q];
  }
  __syncwarp();
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
  const bool ok = cholesky_packed<N, double>(A, lane);
  double x[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    x[q] = i < N ? w.b[i] : 0.0;
  }
  if (ok) chol_subst_f64<N>(A, x, lane);
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    if (i < N) w.F[i] = ok ? (float)x[q] : w.F[i];
  }
  __syncwarp();
  return ok;
}

// One assemble + factorise + solve for the set in w.neg[0..k); refines the
// result when refine == 1.  Returns status flags (0x10 FP64 used, 0x20 the
// FP64 factorisation failed too); bit 0x100 marks that w.W holds no usable
// FP32 factor (the FP64 path ran).
template <int N, bool SPLIT = false, bool PRE = false>
__device__ int assemble_solve(const Scheme& sc, const HTab<N>& H, int k, const WarpWS<N>& w, int lane,
                              float cond_thr, int refine, double* fp64_slot, long long* tacc = nullptr) {
  CSD_T0(t0);
  if constexpr (!PRE) assemble<N, SPLIT>(H, sc.MtMp, k, w, lane);  // PRE: w.W holds Mt_M + G^T G already
  // append b as row N: the factorisation then leaves y = L^-1 b in that row
  {
    float* bN = w.W + packoff(N);
    for (int c = lane; c < packoff(N + 1) - packoff(N); c += 32) bN[c] = c < N ? (float)w.b[c] : 0.f;
    __syncwarp();
  }
  CSD_T1(tacc, kPhAssemble, t0);
  CSD_T0(t1);
  float dmin, dmax;
  const bool ok = cholesky_packed_f32<N>(w.W, w.rdiag, lane, dmin, dmax);
  CSD_T1(tacc, kPhChol, t1);
  const float cond = ok ? (dmax / dmin) * (dmax / dmin) : 3.0e38f;
  if (!ok || !(cond <= cond_thr)) {
    CSD_T0(t2);
    const bool ok64 = solve_fp64<N>(sc, k, w, fp64_slot, lane);
    CSD_T1(tacc, kPhFp64, t2);
    return 0x110 | (ok64 ? 0 : 0x20);
  }
  CSD_T0(t3);
  float x[Dims<N>::CQ];
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    x[q] = i < N ? w.W[packoff(N) + i] : 0.f;
  }
  chol_back_f32<N>(w.W, w.rdiag, x, lane);
#pragma unroll
  for (int q = 0; q < Dims<N>::CQ; ++q) {
    const int i = lane + 32 * q;
    if (i < N) w.F[i] = x[q];
  }
  __syncwarp();
  CSD_T1(tacc, kPhSubst, t3);
  if (refine == 1) {
    CSD_T0(t4);
    refine_step<N>(sc, H, k, w, lane);
    CSD_T1(tacc, kPhRefine, t4);
  }
  return 0;
}

}  // namespace csdb200
