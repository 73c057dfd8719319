// Warm-start network for CSD: a 66 -> 256 -> 256 -> 300 MLP (GELU, sigmoid
// head) that predicts, from a voxel's normalised DW signal, which of the 300
// constraint directions end up in the converged negative set.  BF16
// weights and activations, FP32 accumulation, FP32 master weights and Adam
// moments.  Every step is a hand-written kernel: one tensor-core GEMM
// (mma.sync m16n8k16 bf16, cp.async double buffering, ldmatrix operand
// loads for K-major or MN-major operands) with fused epilogues, plus small
// kernels for input normalisation, the BCE gradient, bias gradients, Adam
// and packing the logits into negative-set bitmasks.
//
// There is no counterpart in MRtrix3: the network only chooses the first
// negative set; the CSD iteration still runs to its own stopping rule.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/csd_b200.h"
#include "umma.cuh"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu: feeds csd_last_error()
// inference kernel of csd_mlp_predict: 0 default, 1 layer-by-layer GEMMs,
// 2 fused tcgen05 (set through csd_set_launch_config)
int g_mlp_infer_kind = 0;
}

namespace {

int mfail(int code, const std::string& m) { return csdb200::set_error(code, m); }
#define MLP_TRY(expr)                                                                         \
  do {                                                                                        \
    cudaError_t e_ = (expr);                                                                  \
    if (e_ != cudaSuccess) return mfail(CSD_ERR_CUDA, std::string(#expr ": ") + cudaGetErrorString(e_)); \
  } while (0)

typedef __nv_bfloat16 bf16;

// ---------------------------------------------------------------------------
// GEMM: C[m][n] = sum_k A(m,k) B(n,k)
//   A(m,k) = A[m*lda + k] (AK) or A[k*lda + m] (!AK)
//   B(n,k) = B[n*ldb + k] (BK) or B[k*ldb + n] (!BK)
// Block tile 128x128x32, 8 warps of 64x32, mma m16n8k16 bf16 -> fp32.
// K-major operands need K % 8 == 0; MN-major operands need M (N) % 8 == 0.

enum Epi { EPI_F32 = 0, EPI_F32_ATOMIC, EPI_BIAS_GELU, EPI_BIAS_F32, EPI_GELU_GRAD };

struct GemmArgs {
  const bf16* A;
  const bf16* B;
  int M, N, K, lda, ldb;
  int kchunk;            // K range per blockIdx.z (split-K)
  float* C32;            // fp32 output (EPI_F32 / EPI_F32_ATOMIC / EPI_BIAS_F32)
  bf16* C16;             // bf16 output (EPI_BIAS_GELU: activation; EPI_GELU_GRAD: gradient)
  bf16* Apre;            // EPI_BIAS_GELU: pre-activation out; EPI_GELU_GRAD: pre-activation in
  const float* bias;
  int ldc;
};

constexpr int BM = 128, BN = 128, BKT = 32;
constexpr int SK = BKT + 8;    // K-major tile row stride (halves)
constexpr int SM = BM + 8;     // MN-major tile row stride (halves)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int Nn>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(Nn));
}
__device__ __forceinline__ void ldsm4(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void ldsm4t(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// Loads one 128x32 (K-major) or 32x128 (MN-major) operand tile with cp.async.
template <bool KMAJ>
__device__ __forceinline__ void load_tile(bf16* s, const bf16* g, int ld, int rows, int K, int r0, int k0) {
  const int t = threadIdx.x;
  if (KMAJ) {
    // 128 rows x 4 chunks of 8 halves
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int id = t + 256 * c;
      const int r = id >> 2, ch = id & 3;
      const int gr = r0 + r, gk = k0 + ch * 8;
      const bool v = gr < rows && gk < K;
      cp_async16(s + r * SK + ch * 8, v ? (g + (long long)gr * ld + gk) : g, v);
    }
  } else {
    // 32 k-rows x 16 chunks of 8 halves (along m)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int id = t + 256 * c;
      const int kr = id >> 4, ch = id & 15;
      const int gk = k0 + kr, gm = r0 + ch * 8;
      const bool v = gk < K && gm < rows;
      cp_async16(s + kr * SM + ch * 8, v ? (g + (long long)gk * ld + gm) : g, v);
    }
  }
}

template <bool AK, bool BK, int EPI>
__global__ void __launch_bounds__(256) gemm_bf16(const GemmArgs a) {
  constexpr int ASZ = AK ? BM * SK : BKT * SM;
  constexpr int BSZ = BK ? BN * SK : BKT * SM;
  __shared__ __align__(16) bf16 sA[2][ASZ];
  __shared__ __align__(16) bf16 sB[2][BSZ];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int kbeg = blockIdx.z * a.kchunk;
  const int kend = min(a.K, kbeg + a.kchunk);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp >> 2) * 64, wn = (warp & 3) * 32;
  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
  const int nk = (kend - kbeg + BKT - 1) / BKT;
  if (nk > 0) {
    load_tile<AK>(sA[0], a.A, a.lda, a.M, kend, m0, kbeg);
    load_tile<BK>(sB[0], a.B, a.ldb, a.N, kend, n0, kbeg);
  }
  cp_commit();
  for (int kt = 0; kt < nk; ++kt) {
    const int cur = kt & 1;
    if (kt + 1 < nk) {
      load_tile<AK>(sA[cur ^ 1], a.A, a.lda, a.M, kend, m0, kbeg + (kt + 1) * BKT);
      load_tile<BK>(sB[cur ^ 1], a.B, a.ldb, a.N, kend, n0, kbeg + (kt + 1) * BKT);
    }
    cp_commit();
    cp_wait<1>();
    __syncthreads();
    const bf16* tA = sA[cur];
    const bf16* tB = sB[cur];
#pragma unroll
    for (int kk = 0; kk < BKT; kk += 16) {
      uint32_t af[4][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int mb = wm + 16 * i;
        if (AK) {
          ldsm4(af[i], tA + (mb + (lane & 15)) * SK + kk + (lane >> 4) * 8);
        } else {
          const int koff = (lane & 7) + ((lane >> 4) << 3), moff = ((lane >> 3) & 1) * 8;
          ldsm4t(af[i], tA + (kk + koff) * SM + mb + moff);
        }
      }
#pragma unroll
      for (int j = 0; j < 4; j += 2) {
        const int nb = wn + 8 * j;
        uint32_t r[4];
        if (BK) {
          const int noff = (lane & 7) + ((lane >> 4) << 3), koff = ((lane >> 3) & 1) * 8;
          ldsm4(r, tB + (nb + noff) * SK + kk + koff);
        } else {
          const int mi = lane >> 3;
          const int koff = (lane & 7) + (mi & 1) * 8, noff = (mi >> 1) * 8;
          ldsm4t(r, tB + (kk + koff) * SM + nb + noff);
        }
        bfr[j][0] = r[0];
        bfr[j][1] = r[1];
        bfr[j + 1][0] = r[2];
        bfr[j + 1][1] = r[3];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bfr[j][0], bfr[j][1]);
    }
    __syncthreads();
  }
  cp_wait<0>();
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int m = m0 + wm + 16 * i + gid + 8 * (e >> 1);
        const int n = n0 + wn + 8 * j + 2 * tig + (e & 1);
        if (m >= a.M || n >= a.N) continue;
        const long long o = (long long)m * a.ldc + n;
        float v = acc[i][j][e];
        if (EPI == EPI_F32) {
          a.C32[o] = v;
        } else if (EPI == EPI_F32_ATOMIC) {
          atomicAdd(a.C32 + o, v);
        } else if (EPI == EPI_BIAS_GELU) {
          v += a.bias[n];
          a.Apre[o] = __float2bfloat16(v);
          a.C16[o] = __float2bfloat16(gelu(v));
        } else if (EPI == EPI_BIAS_F32) {
          a.C32[o] = v + a.bias[n];
        } else if (EPI == EPI_GELU_GRAD) {
          a.C16[o] = __float2bfloat16(v * gelu_grad(__bfloat162float(a.Apre[o])));
        }
      }
}

template <bool AK, bool BK, int EPI>
int gemm(const GemmArgs& a0, int splits, cudaStream_t st) {
  GemmArgs a = a0;
  if (splits < 1) splits = 1;
  a.kchunk = ((a.K + splits - 1) / splits + BKT - 1) / BKT * BKT;
  splits = (a.K + a.kchunk - 1) / a.kchunk;
  dim3 grid((a.N + BN - 1) / BN, (a.M + BM - 1) / BM, splits);
  gemm_bf16<AK, BK, EPI><<<grid, 256, 0, st>>>(a);
  MLP_TRY(cudaGetLastError());
  return 0;
}

// ---------------------------------------------------------------------------
// small kernels

// x[v][t] = (S_t / mean_b0 - mu_t) * inv_sd_t for t < n_in, zero up to ld.
__global__ void mlp_inputs_kernel(const float* dwi, long long n, long long vs, long long ts, int n_in, int ld,
                                  const int* b0, int n_b0, const float* mu, const float* isd, const int* index,
                                  bf16* x) {
  const long long v = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (v >= n) return;
  const float* d = dwi + (index ? (long long)index[v] : v) * vs;
  float s0 = 0.f;
  for (int i = lane; i < n_b0; i += 32) {
    const float x0 = d[(long long)b0[i] * ts];
    s0 += isfinite(x0) ? x0 : 0.f;
  }
  for (int o = 16; o; o >>= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, o);
  s0 = n_b0 ? s0 / n_b0 : 1.f;
  const float inv = s0 > 1e-6f ? 1.f / s0 : 0.f;
  for (int t = lane; t < ld; t += 32) {
    float y = 0.f;
    if (t < n_in) {
      float sv = d[(long long)t * ts];
      sv = isfinite(sv) ? sv : 0.f;
      y = (sv * inv - mu[t]) * isd[t];
    }
    x[v * ld + t] = __float2bfloat16(y);
  }
}

// dZ = (sigmoid(z) - y) / count for the first n_out columns; loss += BCE.
__global__ void mlp_bce_kernel(const float* z, const uint32_t* y, int nw, long long rows, int n_out, int ld,
                               float scale, bf16* dz, float* loss) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < rows * ld) {
    const long long r = i / ld;
    const int c = (int)(i - r * ld);
    float g = 0.f;
    if (c < n_out) {
      const float zz = z[i];
      const float t = ((y[r * nw + (c >> 5)] >> (c & 31)) & 1u) ? 1.f : 0.f;
      const float p = 1.f / (1.f + expf(-zz));
      g = (p - t) * scale;
      // softplus form of the BCE, stable for large |z|
      l = fmaxf(zz, 0.f) - zz * t + log1pf(expf(-fabsf(zz)));
    }
    dz[i] = __float2bfloat16(g);
  }
  for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l * scale);
}

// db[c] += sum_r g[r][c] (fp32 accumulation over a row chunk per block)
__global__ void mlp_colsum_kernel(const bf16* g, long long rows, int cols, int ld, float* db) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  const long long r0 = (long long)blockIdx.y * 256;
  const long long r1 = min(rows, r0 + 256);
  float s = 0.f;
  for (long long r = r0; r < r1; ++r) s += __bfloat162float(g[r * ld + c]);
  atomicAdd(db + c, s);
}

// Adam on fp32 masters; refreshes the bf16 copy.  Parameters live in one
// flat buffer; `ld16`/`rows16` describe where each bf16 weight lands.
__global__ void mlp_adam_kernel(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                                float eps, float c1, float c2, float wd, bf16* w16) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr * ((mi * c1) / (sqrtf(vi * c2) + eps) + wd * w[i]);
  w[i] = wi;
  if (w16) w16[i] = __float2bfloat16(wi);
}

__global__ void mlp_to_bf16_kernel(const float* w, long long n, bf16* w16) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w16[i] = __float2bfloat16(w[i]);
}

// negmask[v][w] bit b = logit[v][32 w + b] > thr (thr = 0: sigmoid > 1/2);
// masked-out voxels get an empty set.
__global__ void mlp_pack_kernel(const float* z, long long rows, int n_out, int ld, int nw, const int* index,
                                float thr, uint32_t* out) {
  const long long r = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  const int lane = threadIdx.x & 31;
  if (r >= rows) return;
  const long long o = (index ? (long long)index[r] : r) * nw;
  for (int w = 0; w < nw; ++w) {
    const int c = 32 * w + lane;
    const uint32_t bits = __ballot_sync(0xffffffffu, c < n_out && z[r * ld + c] > thr);
    if (lane == 0) out[o + w] = bits;
  }
}

// ---------------------------------------------------------------------------
// Fused inference on the 5th-generation tensor cores (sm_100a): one CTA per
// SM walks tiles of 128 voxels; per tile the normalised inputs are built in
// shared memory, the three layers run as tcgen05.mma (M = 128, BF16 operands
// from shared memory, FP32 accumulators in tensor memory: layer 1 in columns
// [0,256), layer 2 in [256,512), the output layer in [0,320)), and 256
// threads run the epilogues straight from tensor memory (bias + GELU back
// into shared memory as the next layer's operand; bias + threshold into
// negative-set bitmasks).  Nothing but the inputs and the bitmasks touches
// HBM.  The weights stream through two shared-memory buffers as nine
// pre-packed slabs (bulk copies completing on mbarriers), the next slab in
// flight while the tensor core works on the current one.  Operands use the
// canonical K-major, non-swizzled layout (8-row x 16-byte core matrices,
// 8-row groups 128 B apart, K chunks of 8 a row-group count x 128 B apart).
// Every wait is bounded; a time-out stops all threads together, drains the
// copies and instructions in flight, frees the tensor memory and raises the
// error flag.
constexpr int kInfRows = 128;
constexpr int kInfThreads = 512;
constexpr int kInfIn = 80;     // padded input width
constexpr int kInfHid = 256;
constexpr int kInfOut = 320;   // padded output width (two N = 160 halves)
constexpr uint32_t kSlabW1 = (kInfIn / 8) * (kInfHid / 8) * 128;  // K 80 x N 256
constexpr uint32_t kSlabW2 = 8 * (kInfHid / 8) * 128;             // K 64 x N 256
constexpr uint32_t kSlabW3 = 8 * (kInfOut / 8) * 128;             // K 64 x N 320
constexpr int kSlabs = 9;                                          // W1, W2 x 4, W3 x 4
constexpr uint32_t kPackedBytes = kSlabW1 + 4 * kSlabW2 + 4 * kSlabW3;
__host__ __device__ constexpr uint32_t inf_slab_off(int j) {
  return j == 0 ? 0u : j <= 4 ? kSlabW1 + (uint32_t)(j - 1) * kSlabW2 : kSlabW1 + 4 * kSlabW2 + (uint32_t)(j - 5) * kSlabW3;
}
__host__ __device__ constexpr uint32_t inf_slab_bytes(int j) { return j == 0 ? kSlabW1 : j <= 4 ? kSlabW2 : kSlabW3; }
constexpr uint32_t kInfX = 0;                                   // [10 chunks][16 groups][8][8] bf16
constexpr uint32_t kInfH = kInfX + (kInfIn / 8) * 2048;          // [32 chunks][16 groups][8][8] bf16
constexpr int kInfBufs = 3;                                      // slab buffers (two copies ahead)
constexpr uint32_t kInfW = kInfH + (kInfHid / 8) * 2048;         // slab buffers
constexpr uint32_t kInfBar = kInfW + kInfBufs * kSlabW3;         // full[3], empty[3], layer, tmem slot
constexpr uint32_t kInfVec = kInfBar + 64;                       // b1, b2, b3, mu, isd (fp32)
constexpr uint32_t kInfSmem = kInfVec + (2 * kInfHid + kInfOut + 2 * kInfIn) * 4;

// Rearranges the BF16 weights into the nine slabs in the core-matrix layout
// (one thread per packed element); rows past n_out and columns past n_in
// of the flat buffer become zero.
__global__ void mlp_pack_tc_kernel(const bf16* w16, long long oW1, long long oW2, long long oW3, int ld_in, int H,
                                   int n_out, bf16* packed) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kPackedBytes / 2) return;
  const uint32_t byte = (uint32_t)i * 2;
  int j = 0;
  while (j + 1 < kSlabs && byte >= inf_slab_off(j + 1)) ++j;
  const uint32_t local = (byte - inf_slab_off(j)) / 2;
  const int nr = j == 0 ? kInfHid : j <= 4 ? kInfHid : kInfOut;  // rows (N) of the slab
  const int e = local & 7, r = (local >> 3) & 7;
  const int cg = local >> 6;                 // core-matrix index: kc * (nr / 8) + ng
  const int kc = cg / (nr / 8), ng = cg - kc * (nr / 8);
  const int n = ng * 8 + r;
  const int k0 = j == 0 ? 0 : 64 * ((j - 1) & 3);
  const int k = k0 + kc * 8 + e;
  bf16 v = __float2bfloat16(0.f);
  if (j == 0) {
    if (k < ld_in) v = w16[oW1 + (long long)n * ld_in + k];
  } else if (j <= 4) {
    v = w16[oW2 + (long long)n * H + k];
  } else if (n < n_out) {
    v = w16[oW3 + (long long)n * H + k];
  }
  packed[i] = v;
}

struct InferArgs {
  const float* dwi;
  long long n, vs, ts;
  const int* index;         // compacted voxel ids or NULL
  const int* b0;
  int n_b0, n_in, n_out, nw;
  const float* mu;
  const float* isd;
  const bf16* packed;
  const float* b1;
  const float* b2;
  const float* b3;
  float thr;
  uint32_t* out;
  int* err;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__global__ void __launch_bounds__(kInfThreads, 1) mlp_infer_tc_kernel(const __grid_constant__ InferArgs a) {
  using namespace csdb200;
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row = 32 * (warp & 3) + lane;   // tensor-memory lane = tile row
  const int qc = warp >> 2;                 // column quarter of the epilogues (4 warps per lane quarter)
  // K chunks of the inputs and words of the output this thread builds: 10
  // of each, split 2 / 3 / 2 / 3 over the quarters
  const int ck0 = (10 * qc) >> 2, ck1 = (10 * (qc + 1)) >> 2;
  const long long ntiles = (a.n + kInfRows - 1) / kInfRows;
  if ((long long)blockIdx.x >= ntiles) return;
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  const uint32_t sX = sbase + kInfX, sH = sbase + kInfH, sW = sbase + kInfW;
  const uint32_t bar = sbase + kInfBar;
  const uint32_t full0 = bar, empty0 = bar + 8 * kInfBufs, layer = bar + 16 * kInfBufs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + kInfBar + 16 * kInfBufs + 8);
  if (tid == 0) {
    for (int b = 0; b < 2 * kInfBufs + 1; ++b) mbar_init(bar + 8 * b, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) tmem_alloc(sbase + kInfBar + 16 * kInfBufs + 8, 512);
  // per-column vectors of the epilogues and the input normalisation
  float* vb1 = reinterpret_cast<float*>(smem + kInfVec);
  float* vb2 = vb1 + kInfHid;
  float* vb3 = vb2 + kInfHid;
  float* vmu = vb3 + kInfOut;
  float* visd = vmu + kInfIn;
  for (int i = tid; i < kInfHid; i += kInfThreads) {
    vb1[i] = a.b1[i];
    vb2[i] = a.b2[i];
  }
  for (int i = tid; i < kInfOut; i += kInfThreads) vb3[i] = i < a.n_out ? a.b3[i] : 0.f;
  for (int i = tid; i < kInfIn; i += kInfThreads) {
    vmu[i] = i < a.n_in ? a.mu[i] : 0.f;
    visd[i] = i < a.n_in ? a.isd[i] : 0.f;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t id256 = umma_idesc_f16(128, 256, true), id160 = umma_idesc_f16(128, 160, true);
  const long long my_tiles = (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x;
  const long long total_slabs = my_tiles * kSlabs;
  // producer / issuer state (thread 0)
  long long g_load = 0;   // slabs whose copy was issued
  long long g_landed = 0; // slabs whose copy was waited for
  bool ok0 = true;
  // slab g lives in buffer g % kInfBufs; the k-th use of a buffer completes
  // its barriers' phase k, of parity k & 1
  auto issue_load = [&](long long g) {
    const int j = (int)(g % kSlabs), b = (int)(g % kInfBufs);
    mbar_arrive_expect_tx(full0 + 8 * b, inf_slab_bytes(j));
    bulk_copy_g2s(sW + b * kSlabW3, reinterpret_cast<const unsigned char*>(a.packed) + inf_slab_off(j),
                  inf_slab_bytes(j), full0 + 8 * b);
    g_load = g + 1;
  };
  // consume slab g: wait for it, issue its instructions, free its buffer on
  // completion, then refill the buffer of slab g - 1 with slab g + 2
  auto consume = [&](long long g, auto&& issue) {
    const int b = (int)(g % kInfBufs);
    if (ok0 && !mbar_wait(full0 + 8 * b, (uint32_t)((g / kInfBufs) & 1))) ok0 = false;
    if (ok0) {
      g_landed = g + 1;
      tc_fence_after();
      issue(sW + b * kSlabW3);
      umma_commit(empty0 + 8 * b);
    }
    if (ok0 && g + 2 < total_slabs) {
      if (g >= 1 && !mbar_wait(empty0 + 8 * ((g - 1) % kInfBufs), (uint32_t)(((g - 1) / kInfBufs) & 1))) ok0 = false;
      if (ok0) issue_load(g + 2);
    }
  };
  if (tid == 0) {
    issue_load(0);
    if (total_slabs > 1) issue_load(1);
  }
  uint32_t lphase = 0;
  long long g = 0;  // next slab to consume
  bool failed = false;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long e0 = tile * kInfRows;
    // ---- inputs: x = (S / mean(S_b0) - mu) * isd.  The tile's raw rows are
    // staged (coalesced, one warp per row) in the H area, free until the
    // first layer's epilogue; each thread then builds columns
    // chunks [ck0, ck1) of its row.
    {
      constexpr int kLdS = kInfIn + 1;  // odd row stride: rows in distinct banks
      constexpr int kRowsPerWarp = kInfRows / (kInfThreads / 32);  // 8
      constexpr int kInChunks = (kInfIn + 31) / 32;                 // 3 samples a lane
      float* Sraw = reinterpret_cast<float*>(smem + kInfH);
      // warp w stages rows w, w + 16, ...: lane j < 8 reads row j's voxel
      // index, then every sample load of the warp's rows is issued before
      // any is stored
      long long vox = -1;
      if (lane < kRowsPerWarp) {
        const long long r = e0 + warp + (kInfThreads / 32) * lane;
        if (r < a.n) vox = a.index ? (long long)a.index[r] : r;
      }
      float xr[kRowsPerWarp][kInChunks];
#pragma unroll
      for (int j = 0; j < kRowsPerWarp; ++j) {
        const long long vj = __shfl_sync(0xffffffffu, vox, j);
        const float* d = a.dwi + (vj < 0 ? 0 : vj) * a.vs;
#pragma unroll
        for (int c = 0; c < kInChunks; ++c) {
          const int t = lane + 32 * c;
          xr[j][c] = (vj >= 0 && t < a.n_in) ? __ldg(d + (long long)t * a.ts) : 0.f;
        }
      }
#pragma unroll
      for (int j = 0; j < kRowsPerWarp; ++j) {
        const int rr = warp + (kInfThreads / 32) * j;
#pragma unroll
        for (int c = 0; c < kInChunks; ++c) {
          const int t = lane + 32 * c;
          if (t < a.n_in) Sraw[rr * kLdS + t] = xr[j][c];
        }
      }
      __syncthreads();
      const long long r = e0 + row;
      float xs[24];
#pragma unroll
      for (int c = 0; c < 24; ++c) xs[c] = 0.f;
      if (r < a.n) {
        const float* sr = Sraw + row * kLdS;
        // mean of the b=0 samples, summed in the order of mlp_inputs_kernel
        float part[32];
#pragma unroll
        for (int l = 0; l < 32; ++l) part[l] = 0.f;
        for (int i = 0; i < a.n_b0; ++i) {
          const float x0 = sr[a.b0[i]];
          part[i & 31] += isfinite(x0) ? x0 : 0.f;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1)
#pragma unroll
          for (int l = 0; l < o; ++l) part[l] = part[l] + part[l + o];
        const float s0 = a.n_b0 ? part[0] / a.n_b0 : 1.f;
        const float inv = s0 > 1e-6f ? 1.f / s0 : 0.f;
#pragma unroll
        for (int c = 0; c < 24; ++c) {
          const int t = 8 * ck0 + c;
          if (t < 8 * ck1 && t < a.n_in) {
            float sv = sr[t];
            sv = isfinite(sv) ? sv : 0.f;
            xs[c] = (sv * inv - vmu[t]) * visd[t];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int kc = ck0 + q;
        if (kc >= ck1) break;
        uint4 u;
        u.x = pack_bf16x2(xs[8 * q], xs[8 * q + 1]);
        u.y = pack_bf16x2(xs[8 * q + 2], xs[8 * q + 3]);
        u.z = pack_bf16x2(xs[8 * q + 4], xs[8 * q + 5]);
        u.w = pack_bf16x2(xs[8 * q + 6], xs[8 * q + 7]);
        *reinterpret_cast<uint4*>(smem + kInfX + kc * 2048 + (row >> 3) * 128 + (row & 7) * 16) = u;
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    // ---- three layers: instructions (thread 0), then the epilogue (all)
#pragma unroll 1
    for (int L = 0; L < 3; ++L) {
      if (tid == 0) {
        tc_fence_after();
        const int nsl = L == 0 ? 1 : 4;
        for (int sl = 0; sl < nsl; ++sl, ++g) {
          if (L == 0) {
            consume(g, [&](uint32_t wb) {
#pragma unroll
              for (int ks = 0; ks < kInfIn / 16; ++ks)
                umma_f16_ss(tmem, umma_smem_desc(sX + 2 * ks * 2048, 2048, 128),
                            umma_smem_desc(wb + 2 * ks * (kInfHid / 8) * 128, (kInfHid / 8) * 128, 128), id256,
                            ks > 0);
            });
          } else if (L == 1) {
            consume(g, [&](uint32_t wb) {
#pragma unroll
              for (int ks = 0; ks < 4; ++ks)
                umma_f16_ss(tmem + 256, umma_smem_desc(sH + (8 * sl + 2 * ks) * 2048, 2048, 128),
                            umma_smem_desc(wb + 2 * ks * (kInfHid / 8) * 128, (kInfHid / 8) * 128, 128), id256,
                            (sl | ks) != 0);
            });
          } else {
            consume(g, [&](uint32_t wb) {
#pragma unroll
              for (int ks = 0; ks < 4; ++ks)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                  umma_f16_ss(tmem + 160 * h, umma_smem_desc(sH + (8 * sl + 2 * ks) * 2048, 2048, 128),
                              umma_smem_desc(wb + 2 * ks * (kInfOut / 8) * 128 + h * (160 / 8) * 128,
                                             (kInfOut / 8) * 128, 128),
                              id160, (sl | ks) != 0);
            });
          }
        }
        umma_commit(layer);  // also when stopping: lets the other threads reach the vote
      }
      bool okw = (tid != 0 || ok0) && mbar_wait(layer, lphase);
      lphase ^= 1u;
      if (!__syncthreads_and(okw)) {
        failed = true;
        break;
      }
      tc_fence_after();
      const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
      if (L < 2) {
        // bias + GELU -> BF16 -> the next layer's A operand (columns [64 qc, 64 qc + 64))
        const float* bias = L == 0 ? vb1 : vb2;
#pragma unroll 1
        for (int jj = 0; jj < 4; jj += 2) {
          uint32_t v2[2][16];
          tmem_ld16(lane_base + (uint32_t)(256 * L + 64 * qc + 16 * jj), v2[0]);
          tmem_ld16(lane_base + (uint32_t)(256 * L + 64 * qc + 16 * jj + 16), v2[1]);
          tmem_ld_wait();
#pragma unroll
          for (int u = 0; u < 2; ++u) {
          const int c0 = 64 * qc + 16 * (jj + u);
          const uint32_t* v = v2[u];
          float y[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) y[e] = gelu(__uint_as_float(v[e]) + bias[c0 + e]);
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            uint4 u;
            u.x = pack_bf16x2(y[8 * q], y[8 * q + 1]);
            u.y = pack_bf16x2(y[8 * q + 2], y[8 * q + 3]);
            u.z = pack_bf16x2(y[8 * q + 4], y[8 * q + 5]);
            u.w = pack_bf16x2(y[8 * q + 6], y[8 * q + 7]);
            const int kc = c0 / 8 + q;
            *reinterpret_cast<uint4*>(smem + kInfH + kc * 2048 + (row >> 3) * 128 + (row & 7) * 16) = u;
          }
          }
        }
        fence_async_smem();
      } else {
        // bias + threshold -> negative-set bits (words [ck0, ck1) of the 10)
        const long long r = e0 + row;
        uint32_t words[3] = {0u, 0u, 0u};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (ck0 + k >= ck1) break;  // uniform over the warp
          const int c0 = 32 * (ck0 + k);
          uint32_t v2[2][16];
          tmem_ld16(lane_base + (uint32_t)c0, v2[0]);
          tmem_ld16(lane_base + (uint32_t)(c0 + 16), v2[1]);
          tmem_ld_wait();
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              const int c = c0 + 16 * u + e;
              if (c < a.n_out && __uint_as_float(v2[u][e]) + vb3[c] > a.thr) words[k] |= 1u << (c & 31);
            }
        }
        if (r < a.n) {
          const long long o = (a.index ? (long long)a.index[r] : r) * a.nw;
#pragma unroll
          for (int k = 0; k < 3; ++k)
            if (ck0 + k < ck1 && ck0 + k < a.nw) a.out[o + ck0 + k] = words[k];
        }
      }
      tc_fence_before();
      __syncthreads();
    }
    if (failed) break;
  }
  if (failed && tid == 0) {
    // drain: the copies still in flight, the pending layer commit, then a
    // fresh commit that completes once every issued instruction is done
    for (long long q = g_landed; q < g_load; ++q)
      mbar_wait(full0 + 8 * (q % kInfBufs), (uint32_t)((q / kInfBufs) & 1));
    mbar_wait(layer, lphase ^ 1u);
    umma_commit(layer);
    mbar_wait(layer, lphase);
    atomicExch(a.err, 1);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, 512);
}

// index[] = positions of the voxels with mask != 0 (order not preserved)
__global__ void mlp_compact_kernel(const uint8_t* mask, long long n, int* index, int* count) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const bool on = i < n && mask[i];
  const unsigned b = __ballot_sync(0xffffffffu, on);
  int base = 0;
  if ((threadIdx.x & 31) == 0 && b) base = atomicAdd(count, __popc(b));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (on) index[base + __popc(b & ((1u << (threadIdx.x & 31)) - 1u))] = (int)i;
}

}  // namespace

// ---------------------------------------------------------------------------
// model

struct csd_mlp {
  int n_in = 0, n_hid = 0, n_out = 0;
  int ld_in = 0, ld_out = 0;   // padded widths (multiples of 8)
  int nw = 0;
  int device = 0;
  long long n_params = 0;
  // flat fp32 masters [W1 b1 W2 b2 W3 b3], gradients, Adam moments
  float* w = nullptr;
  float* g = nullptr;
  float* am = nullptr;
  float* av = nullptr;
  bf16* w16 = nullptr;         // bf16 copy of the whole flat buffer (biases unused)
  long long oW1, ob1, oW2, ob2, oW3, ob3;
  long long step = 0;
  // input normalisation
  std::vector<int> b0_host;
  int* b0 = nullptr;
  float* mu = nullptr;
  float* isd = nullptr;
  // activations for up to `cap` rows
  long long cap = 0;
  bf16 *x = nullptr, *a1 = nullptr, *h1 = nullptr, *a2 = nullptr, *h2 = nullptr, *dz = nullptr, *da2 = nullptr,
       *da1 = nullptr;
  float* z = nullptr;
  float* loss = nullptr;
  int* idx = nullptr;          // compacted voxel index list for masked prediction
  long long idx_cap = 0;
  // fused inference: weights packed into slabs, refreshed when they change
  bf16* wpack = nullptr;
  long long wver = 1, pver = 0;
  int* err = nullptr;          // device time-out flag of the fused kernel
};

static int mlp_reserve(csd_mlp* m, long long rows) {
  if (rows <= m->cap) return 0;
  cudaFree(m->x);
  cudaFree(m->a1);
  cudaFree(m->h1);
  cudaFree(m->a2);
  cudaFree(m->h2);
  cudaFree(m->dz);
  cudaFree(m->da2);
  cudaFree(m->da1);
  cudaFree(m->z);
  const long long R = (rows + 127) / 128 * 128;
  MLP_TRY(cudaMalloc(&m->x, R * m->ld_in * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->a1, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->h1, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->a2, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->h2, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->dz, R * m->ld_out * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->da2, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->da1, R * m->n_hid * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->z, R * m->ld_out * sizeof(float)));
  m->cap = R;
  return 0;
}

extern "C" int csd_mlp_create(int n_in, int n_hidden, int n_out, uint64_t seed, csd_mlp** out) {
  if (!out || n_in <= 0 || n_hidden <= 0 || n_out <= 0 || n_hidden % 8 || n_out > 512)
    return mfail(CSD_ERR_INVALID, "csd_mlp_create: invalid sizes (n_hidden must be a multiple of 8)");
  *out = nullptr;
  std::unique_ptr<csd_mlp> m(new csd_mlp);
  m->n_in = n_in;
  m->n_hid = n_hidden;
  m->n_out = n_out;
  m->ld_in = (n_in + 15) / 16 * 16;
  m->ld_out = (n_out + 7) / 8 * 8;
  m->nw = (n_out + 31) / 32;
  MLP_TRY(cudaGetDevice(&m->device));
  // layout of the flat parameter buffer; weights are [out][in_padded]
  long long o = 0;
  m->oW1 = o; o += (long long)n_hidden * m->ld_in;
  m->ob1 = o; o += n_hidden;
  m->oW2 = o; o += (long long)n_hidden * n_hidden;
  m->ob2 = o; o += n_hidden;
  m->oW3 = o; o += (long long)m->ld_out * n_hidden;
  m->ob3 = o; o += m->ld_out;
  m->n_params = o;
  std::vector<float> h((size_t)o, 0.f);
  std::mt19937_64 rng(seed);
  auto init = [&](long long off, int rows, int cols, int ld, int fan_in) {
    const float lim = 1.0f / std::sqrt((float)fan_in);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (int r = 0; r < rows; ++r)
      for (int c = 0; c < cols; ++c) h[(size_t)(off + (long long)r * ld + c)] = U(rng);
  };
  init(m->oW1, n_hidden, n_in, m->ld_in, n_in);
  init(m->oW2, n_hidden, n_hidden, n_hidden, n_hidden);
  init(m->oW3, n_out, n_hidden, n_hidden, n_hidden);
  MLP_TRY(cudaMalloc(&m->w, o * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->g, o * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->am, o * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->av, o * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->w16, o * sizeof(bf16)));
  MLP_TRY(cudaMalloc(&m->mu, m->ld_in * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->isd, m->ld_in * sizeof(float)));
  MLP_TRY(cudaMalloc(&m->loss, sizeof(float)));
  MLP_TRY(cudaMemcpy(m->w, h.data(), o * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemset(m->am, 0, o * sizeof(float)));
  MLP_TRY(cudaMemset(m->av, 0, o * sizeof(float)));
  std::vector<float> mu(m->ld_in, 0.f), isd(m->ld_in, 1.f);
  MLP_TRY(cudaMemcpy(m->mu, mu.data(), mu.size() * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(m->isd, isd.data(), isd.size() * sizeof(float), cudaMemcpyHostToDevice));
  mlp_to_bf16_kernel<<<(unsigned)((o + 255) / 256), 256>>>(m->w, o, m->w16);
  MLP_TRY(cudaGetLastError());
  MLP_TRY(cudaDeviceSynchronize());
  *out = m.release();
  return CSD_OK;
}

extern "C" void csd_mlp_destroy(csd_mlp* m) {
  if (!m) return;
  void* ps[] = {m->w, m->g, m->am, m->av, m->w16, m->b0, m->mu, m->isd, m->x, m->a1, m->h1, m->a2, m->h2,
                m->dz, m->da2, m->da1, m->z, m->loss, m->idx, m->wpack, m->err};
  for (void* p : ps) cudaFree(p);
  delete m;
}

extern "C" int64_t csd_mlp_param_count(const csd_mlp* m) { return m ? m->n_params : -1; }

extern "C" int csd_mlp_get_params(const csd_mlp* m, float* out, int64_t n) {
  if (!m || !out || n != m->n_params) return mfail(CSD_ERR_INVALID, "csd_mlp_get_params: size mismatch");
  MLP_TRY(cudaMemcpy(out, m->w, n * sizeof(float), cudaMemcpyDeviceToHost));
  return CSD_OK;
}

extern "C" int csd_mlp_set_params(csd_mlp* m, const float* in, int64_t n) {
  if (!m || !in || n != m->n_params) return mfail(CSD_ERR_INVALID, "csd_mlp_set_params: size mismatch");
  MLP_TRY(cudaMemcpy(m->w, in, n * sizeof(float), cudaMemcpyHostToDevice));
  mlp_to_bf16_kernel<<<(unsigned)((n + 255) / 256), 256>>>(m->w, n, m->w16);
  MLP_TRY(cudaGetLastError());
  MLP_TRY(cudaDeviceSynchronize());
  ++m->wver;
  return CSD_OK;
}

extern "C" int csd_mlp_set_inputs(csd_mlp* m, const int* b0_index, int n_b0, const float* mean, const float* stdev) {
  if (!m || n_b0 < 0 || (n_b0 && !b0_index) || !mean || !stdev)
    return mfail(CSD_ERR_INVALID, "csd_mlp_set_inputs: invalid argument");
  for (int i = 0; i < n_b0; ++i)
    if (b0_index[i] < 0 || b0_index[i] >= m->n_in)
      return mfail(CSD_ERR_INVALID, "csd_mlp_set_inputs: b=0 volume index out of range");
  std::vector<float> mu(m->ld_in, 0.f), isd(m->ld_in, 0.f);
  for (int t = 0; t < m->n_in; ++t) {
    mu[t] = mean[t];
    isd[t] = stdev[t] > 0.f ? 1.f / stdev[t] : 0.f;
  }
  MLP_TRY(cudaMemcpy(m->mu, mu.data(), mu.size() * sizeof(float), cudaMemcpyHostToDevice));
  MLP_TRY(cudaMemcpy(m->isd, isd.data(), isd.size() * sizeof(float), cudaMemcpyHostToDevice));
  cudaFree(m->b0);
  m->b0 = nullptr;
  m->b0_host.assign(b0_index, b0_index + n_b0);
  MLP_TRY(cudaMalloc(&m->b0, std::max(1, n_b0) * sizeof(int)));
  if (n_b0) MLP_TRY(cudaMemcpy(m->b0, b0_index, n_b0 * sizeof(int), cudaMemcpyHostToDevice));
  return CSD_OK;
}

static int mlp_inputs(const csd_mlp* m, const float* dwi, long long n, long long vs, long long ts, bf16* x,
                      cudaStream_t st, const int* index = nullptr) {
  if (n <= 0) return 0;
  mlp_inputs_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(dwi, n, vs, ts, m->n_in, m->ld_in, m->b0,
                                                            (int)m->b0_host.size(), m->mu, m->isd, index, x);
  MLP_TRY(cudaGetLastError());
  return 0;
}

extern "C" int csd_mlp_inputs(const csd_mlp* m, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                              int64_t volume_stride, uint16_t* x, void* stream) {
  if (!m || (n_voxels > 0 && (!dwi || !x)) || !m->b0) return mfail(CSD_ERR_INVALID, "csd_mlp_inputs: invalid argument");
  return mlp_inputs(m, dwi, n_voxels, voxel_stride, volume_stride, reinterpret_cast<bf16*>(x),
                    static_cast<cudaStream_t>(stream));
}

// forward for rows [0, n) of x; logits land in m->z
static int mlp_forward(const csd_mlp* m, const bf16* x, long long n, cudaStream_t st) {
  GemmArgs a{};
  a.A = x; a.B = m->w16 + m->oW1; a.M = (int)n; a.N = m->n_hid; a.K = m->ld_in; a.lda = m->ld_in; a.ldb = m->ld_in;
  a.C16 = m->h1; a.Apre = m->a1; a.bias = m->w + m->ob1; a.ldc = m->n_hid;
  int rc = gemm<true, true, EPI_BIAS_GELU>(a, 1, st);
  if (rc) return rc;
  a = GemmArgs{};
  a.A = m->h1; a.B = m->w16 + m->oW2; a.M = (int)n; a.N = m->n_hid; a.K = m->n_hid; a.lda = m->n_hid; a.ldb = m->n_hid;
  a.C16 = m->h2; a.Apre = m->a2; a.bias = m->w + m->ob2; a.ldc = m->n_hid;
  if ((rc = gemm<true, true, EPI_BIAS_GELU>(a, 1, st))) return rc;
  a = GemmArgs{};
  a.A = m->h2; a.B = m->w16 + m->oW3; a.M = (int)n; a.N = m->ld_out; a.K = m->n_hid; a.lda = m->n_hid; a.ldb = m->n_hid;
  a.C32 = m->z; a.bias = m->w + m->ob3; a.ldc = m->ld_out;
  return gemm<true, true, EPI_BIAS_F32>(a, 1, st);
}

// loss + gradients for rows [0, n) of x with targets y; grads land in m->g
static int mlp_backward(csd_mlp* m, const bf16* x, const uint32_t* y, long long n, cudaStream_t st) {
  MLP_TRY(cudaMemsetAsync(m->g, 0, m->n_params * sizeof(float), st));
  const float scale = 1.0f / ((float)n * (float)m->n_out);
  const long long tot = n * m->ld_out;
  mlp_bce_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(m->z, y, m->nw, n, m->n_out, m->ld_out, scale, m->dz,
                                                                  m->loss);
  MLP_TRY(cudaGetLastError());
  const int splits = (int)std::max<long long>(1, std::min<long long>(64, n / 512));
  const int H = m->n_hid;
  // dW3 = dZ^T H2, db3 = colsum(dZ)
  GemmArgs a{};
  a.A = m->dz; a.B = m->h2; a.M = m->ld_out; a.N = H; a.K = (int)n; a.lda = m->ld_out; a.ldb = H;
  a.C32 = m->g + m->oW3; a.ldc = H;
  int rc = gemm<false, false, EPI_F32_ATOMIC>(a, splits, st);
  if (rc) return rc;
  mlp_colsum_kernel<<<dim3((m->ld_out + 127) / 128, (unsigned)((n + 255) / 256)), 128, 0, st>>>(m->dz, n, m->ld_out,
                                                                                               m->ld_out, m->g + m->ob3);
  // dA2 = (dZ W3) * gelu'(A2)
  a = GemmArgs{};
  a.A = m->dz; a.B = m->w16 + m->oW3; a.M = (int)n; a.N = H; a.K = m->ld_out; a.lda = m->ld_out; a.ldb = H;
  a.C16 = m->da2; a.Apre = m->a2; a.ldc = H;
  if ((rc = gemm<true, false, EPI_GELU_GRAD>(a, 1, st))) return rc;
  // dW2 = dA2^T H1, db2
  a = GemmArgs{};
  a.A = m->da2; a.B = m->h1; a.M = H; a.N = H; a.K = (int)n; a.lda = H; a.ldb = H; a.C32 = m->g + m->oW2; a.ldc = H;
  if ((rc = gemm<false, false, EPI_F32_ATOMIC>(a, splits, st))) return rc;
  mlp_colsum_kernel<<<dim3((H + 127) / 128, (unsigned)((n + 255) / 256)), 128, 0, st>>>(m->da2, n, H, H, m->g + m->ob2);
  // dA1 = (dA2 W2) * gelu'(A1)
  a = GemmArgs{};
  a.A = m->da2; a.B = m->w16 + m->oW2; a.M = (int)n; a.N = H; a.K = H; a.lda = H; a.ldb = H;
  a.C16 = m->da1; a.Apre = m->a1; a.ldc = H;
  if ((rc = gemm<true, false, EPI_GELU_GRAD>(a, 1, st))) return rc;
  // dW1 = dA1^T X, db1
  a = GemmArgs{};
  a.A = m->da1; a.B = x; a.M = H; a.N = m->ld_in; a.K = (int)n; a.lda = H; a.ldb = m->ld_in;
  a.C32 = m->g + m->oW1; a.ldc = m->ld_in;
  if ((rc = gemm<false, false, EPI_F32_ATOMIC>(a, splits, st))) return rc;
  mlp_colsum_kernel<<<dim3((H + 127) / 128, (unsigned)((n + 255) / 256)), 128, 0, st>>>(m->da1, n, H, H, m->g + m->ob1);
  MLP_TRY(cudaGetLastError());
  return 0;
}

extern "C" int csd_mlp_gradients(csd_mlp* m, const uint16_t* x, const uint32_t* negmask, int64_t n, float* grad_out,
                                 float* loss_out) {
  if (!m || !x || !negmask || n <= 0 || !grad_out) return mfail(CSD_ERR_INVALID, "csd_mlp_gradients: invalid argument");
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  MLP_TRY(cudaMemset(m->loss, 0, sizeof(float)));
  if ((rc = mlp_forward(m, reinterpret_cast<const bf16*>(x), n, 0))) return rc;
  if ((rc = mlp_backward(m, reinterpret_cast<const bf16*>(x), negmask, n, 0))) return rc;
  MLP_TRY(cudaDeviceSynchronize());
  MLP_TRY(cudaMemcpy(grad_out, m->g, m->n_params * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss_out) MLP_TRY(cudaMemcpy(loss_out, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return CSD_OK;
}

extern "C" int csd_mlp_logits(csd_mlp* m, const uint16_t* x, int64_t n, float* z_out) {
  if (!m || !x || n <= 0 || !z_out) return mfail(CSD_ERR_INVALID, "csd_mlp_logits: invalid argument");
  int rc = mlp_reserve(m, n);
  if (rc) return rc;
  if ((rc = mlp_forward(m, reinterpret_cast<const bf16*>(x), n, 0))) return rc;
  MLP_TRY(cudaDeviceSynchronize());
  MLP_TRY(cudaMemcpy(z_out, m->z, n * m->ld_out * sizeof(float), cudaMemcpyDeviceToHost));
  return CSD_OK;
}

// One pass over the training rows in shuffled mini-batches with Adam.
extern "C" int csd_mlp_train_epoch(csd_mlp* m, const uint16_t* x, const uint32_t* negmask, int64_t n, int batch,
                                   float lr, float weight_decay, uint64_t seed, float* mean_loss, void* stream) {
  if (!m || !x || !negmask || n <= 0 || batch <= 0 || batch % 128)
    return mfail(CSD_ERR_INVALID, "csd_mlp_train_epoch: invalid argument (batch must be a multiple of 128)");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = mlp_reserve(m, batch);
  if (rc) return rc;
  const bf16* X = reinterpret_cast<const bf16*>(x);
  // batches are contiguous row blocks visited in a seeded random order (the
  // caller shuffles the rows once; this keeps every batch a plain slice)
  const long long nb = n / batch;
  std::vector<long long> order(nb);
  for (long long i = 0; i < nb; ++i) order[i] = i;
  std::mt19937_64 rng(seed);
  std::shuffle(order.begin(), order.end(), rng);
  MLP_TRY(cudaMemsetAsync(m->loss, 0, sizeof(float), st));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (long long bi = 0; bi < nb; ++bi) {
    const long long r0 = order[bi] * batch;
    if ((rc = mlp_forward(m, X + r0 * m->ld_in, batch, st))) return rc;
    if ((rc = mlp_backward(m, X + r0 * m->ld_in, negmask + r0 * m->nw, batch, st))) return rc;
    ++m->step;
    const float c1 = 1.f / (1.f - std::pow(b1, (float)m->step));
    const float c2 = 1.f / (1.f - std::pow(b2, (float)m->step));
    mlp_adam_kernel<<<(unsigned)((m->n_params + 255) / 256), 256, 0, st>>>(m->w, m->g, m->am, m->av, m->n_params, lr,
                                                                           b1, b2, eps, c1, c2, weight_decay, m->w16);
    MLP_TRY(cudaGetLastError());
  }
  ++m->wver;
  if (mean_loss) {
    float l = 0.f;
    MLP_TRY(cudaMemcpyAsync(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost, st));
    MLP_TRY(cudaStreamSynchronize(st));
    *mean_loss = nb ? l / (float)nb : 0.f;
  }
  return CSD_OK;
}

// Predicted first negative sets for n voxels of a DWI volume (device).  With
// a mask, only the voxels inside it go through the network (the others get
// an empty set).
// csd_mlp_predict's fused path over n rows (compacted through index when
// it is not NULL); synchronises the stream to read the time-out flag.
static int mlp_predict_fused(csd_mlp* m, const float* dwi, long long n, long long vs, long long ts, const int* index,
                             float thr, uint32_t* negmask, cudaStream_t st) {
  if (!m->wpack) MLP_TRY(cudaMalloc(&m->wpack, kPackedBytes));
  if (!m->err) MLP_TRY(cudaMalloc(&m->err, sizeof(int)));
  if (m->pver != m->wver) {
    mlp_pack_tc_kernel<<<(kPackedBytes / 2 + 255) / 256, 256, 0, st>>>(m->w16, m->oW1, m->oW2, m->oW3, m->ld_in,
                                                                       m->n_hid, m->n_out, m->wpack);
    MLP_TRY(cudaGetLastError());
    m->pver = m->wver;
  }
  if (n <= 0) return CSD_OK;
  int dev = 0, nsm = 0;
  MLP_TRY(cudaGetDevice(&dev));
  MLP_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  MLP_TRY(cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInfSmem));
  MLP_TRY(cudaMemsetAsync(m->err, 0, sizeof(int), st));
  InferArgs a{};
  a.dwi = dwi;
  a.n = n;
  a.vs = vs;
  a.ts = ts;
  a.index = index;
  a.b0 = m->b0;
  a.n_b0 = (int)m->b0_host.size();
  a.n_in = m->n_in;
  a.n_out = m->n_out;
  a.nw = m->nw;
  a.mu = m->mu;
  a.isd = m->isd;
  a.packed = m->wpack;
  a.b1 = m->w + m->ob1;
  a.b2 = m->w + m->ob2;
  a.b3 = m->w + m->ob3;
  a.thr = thr;
  a.out = negmask;
  a.err = m->err;
  const long long tiles = (n + kInfRows - 1) / kInfRows;
  mlp_infer_tc_kernel<<<(unsigned)std::min<long long>(tiles, nsm), kInfThreads, kInfSmem, st>>>(a);
  MLP_TRY(cudaGetLastError());
  int err = 0;
  MLP_TRY(cudaMemcpyAsync(&err, m->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MLP_TRY(cudaStreamSynchronize(st));
  if (err) return mfail(CSD_ERR_TIMEOUT, "csd_mlp_predict: a bounded wait on the tensor cores timed out");
  return CSD_OK;
}

extern "C" int csd_mlp_predict(csd_mlp* m, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                               int64_t volume_stride, const uint8_t* mask, float logit_threshold, uint32_t* negmask,
                               void* stream) {
  if (!m || n_voxels < 0 || (n_voxels > 0 && (!dwi || !negmask)) || !m->b0)
    return mfail(CSD_ERR_INVALID, "csd_mlp_predict: invalid argument (inputs not configured?)");
  if (n_voxels == 0) return CSD_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int kind = csdb200::g_mlp_infer_kind ? csdb200::g_mlp_infer_kind : 2;
  const bool fused = kind == 2 && m->n_hid == kInfHid && m->ld_in <= kInfIn && m->ld_out <= kInfOut;
  const long long chunk = 1 << 18;
  int rc = fused ? 0 : mlp_reserve(m, std::min<long long>(chunk, n_voxels));
  if (rc) return rc;
  const int* index = nullptr;
  long long n = n_voxels;
  if (mask) {
    if (m->idx_cap < n_voxels) {
      cudaFree(m->idx);
      m->idx = nullptr;
      m->idx_cap = 0;
      MLP_TRY(cudaMalloc(&m->idx, (n_voxels + 1) * sizeof(int)));
      m->idx_cap = n_voxels;
    }
    MLP_TRY(cudaMemsetAsync(m->idx + n_voxels, 0, sizeof(int), st));
    mlp_compact_kernel<<<(unsigned)((n_voxels + 255) / 256), 256, 0, st>>>(mask, n_voxels, m->idx, m->idx + n_voxels);
    MLP_TRY(cudaGetLastError());
    int cnt = 0;
    MLP_TRY(cudaMemcpyAsync(&cnt, m->idx + n_voxels, sizeof(int), cudaMemcpyDeviceToHost, st));
    MLP_TRY(cudaMemsetAsync(negmask, 0, (size_t)n_voxels * m->nw * sizeof(uint32_t), st));
    MLP_TRY(cudaStreamSynchronize(st));
    index = m->idx;
    n = cnt;
  }
  if (fused) return mlp_predict_fused(m, dwi, n, voxel_stride, volume_stride, index, logit_threshold, negmask, st);
  for (long long a = 0; a < n; a += chunk) {
    const long long c = std::min<long long>(chunk, n - a);
    if (index) {
      if ((rc = mlp_inputs(m, dwi, c, voxel_stride, volume_stride, m->x, st, index + a))) return rc;
    } else {
      if ((rc = mlp_inputs(m, dwi + a * voxel_stride, c, voxel_stride, volume_stride, m->x, st))) return rc;
    }
    if ((rc = mlp_forward(m, m->x, c, st))) return rc;
    mlp_pack_kernel<<<(unsigned)((c + 7) / 8), 256, 0, st>>>(m->z, c, m->n_out, m->ld_out, m->nw,
                                                             index ? index + a : nullptr, logit_threshold,
                                                             index ? negmask : negmask + a * m->nw);
    MLP_TRY(cudaGetLastError());
  }
  return CSD_OK;
}
