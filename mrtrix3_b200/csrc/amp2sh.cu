// amp2sh on the GPU: the least-squares SH fit of amplitudes sampled along a
// set of directions (MRtrix3 cmd/amp2sh.cpp:108-127, 153-171), per voxel
// c = pinv(SH2amp) a with a = the voxel's amplitudes of the selected volumes,
// optionally scaled by nb0 / (1 + sum of its b=0 amplitudes) (get_amps,
// amp2sh.cpp:157-168, with the reference's initial 1).  In FP64 like the
// reference; the output is float.
//
// The fit is FP64-bound (2 nSH nd flops against 4 (nd + nb0 + nSH) bytes a
// voxel: 5400 flops / 444 B at lmax 8 with 60 directions).  The tile kernel
// keeps the whole fit matrix in shared memory for the life of a persistent
// block, transposed to [nd][columns] so that lane l reads columns l, l + 32,
// ...; a block stages 64 voxels' scaled amplitudes, and each warp forms 8
// voxels x all columns with the products in registers (the voxel's
// amplitudes are broadcast loads).  Fits whose matrix does not fit in shared
// memory take the row kernel: 32 voxels staged, one dot product a thread.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/csd_b200.h"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu
// amp2sh kernel: 0 the fastest that applies, 1 row, 2 tile (FP64 FMA),
// 3 FP64 tensor cores (where they apply); set by csd_set_launch_config
int g_amp2sh_kind = 0;
}

namespace {

constexpr int kA2sRows = 32;
constexpr int kA2sThreads = 256;
constexpr int kA2sMaxDirs = 800;  // the row kernel stages 32 x (nd + 1) doubles

struct Amp2ShArgs {
  const float* amp;
  long long n, vs, ts;
  const double* fit;  // [nsh][nd]
  const int* dwis;    // [nd]
  const int* b0;      // [nb0] or NULL
  int nd, nb0, nsh, normalise;
  int contig;      // tensor-core kernel: volume stride 1 and 16-byte aligned rows
  int row_floats;  // tensor-core kernel: staged floats a voxel
  float* out;
  long long os;
};

__global__ void __launch_bounds__(kA2sThreads) amp2sh_kernel(const __grid_constant__ Amp2ShArgs a) {
  extern __shared__ __align__(16) double asm_[];
  const int lda = a.nd + 1;
  double* A = asm_;  // [kA2sRows][lda]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long ntiles = (a.n + kA2sRows - 1) / kA2sRows;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long v0 = tile * kA2sRows;
    __syncthreads();
    for (int r = warp; r < kA2sRows; r += kA2sThreads / 32) {
      const long long v = v0 + r;
      if (v >= a.n) break;
      const float* p = a.amp + v * a.vs;
      double norm = 1.0;
      if (a.normalise) {
        // get_amps' sum, in its order: 1 + the b=0 amplitudes one by one
        double s = 1.0;
        for (int i = 0; i < a.nb0; ++i) s += (double)p[(long long)a.b0[i] * a.ts];
        norm = (double)a.nb0 / s;
      }
      for (int t = lane; t < a.nd; t += 32) A[r * lda + t] = (double)p[(long long)a.dwis[t] * a.ts] * norm;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kA2sRows * a.nsh; i += blockDim.x) {
      const int r = i / a.nsh, c = i - r * a.nsh;
      const long long v = v0 + r;
      if (v >= a.n) continue;
      const double* f = a.fit + (long long)c * a.nd;
      const double* x = A + r * lda;
      double s0 = 0.0, s1 = 0.0;
      int t = 0;
      for (; t + 1 < a.nd; t += 2) {
        s0 = fma(__ldg(f + t), x[t], s0);
        s1 = fma(__ldg(f + t + 1), x[t + 1], s1);
      }
      if (t < a.nd) s0 = fma(__ldg(f + t), x[t], s0);
      a.out[v * a.os + c] = (float)(s0 + s1);
    }
  }
}

constexpr int kTileWarps = 8;
constexpr int kTileVox = 8;  // voxels a warp forms
constexpr int kTileRows = kTileWarps * kTileVox;

// Shared-memory layout of the tile kernel: F [ndp][32 JC] transposed fit
// (rows nd.. ndp-1 zero) and A [kTileRows][ndp] scaled amplitudes, in double
// (ndp = nd rounded up to even, so that a voxel's pair k, k+1 is one 16-byte
// load); then the float staging of the next tile, Af [kTileRows][ndp] and
// Bf [kTileRows][nb0] (its b=0 amplitudes), and the volume indices.
__host__ __device__ inline int tile_ndp(int nd) { return (nd + 1) & ~1; }
__host__ inline size_t tile_smem_bytes(int nd, int nb0, int jc) {
  const size_t ndp = (size_t)tile_ndp(nd);
  return (ndp * 32 * jc + (size_t)kTileRows * ndp) * sizeof(double) +
         ((size_t)kTileRows * (ndp + nb0) + nd + nb0) * sizeof(float);
}

__device__ __forceinline__ void cp_async4(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

template <int JC>
__global__ void __launch_bounds__(kTileWarps * 32, 2) amp2sh_tile_kernel(const __grid_constant__ Amp2ShArgs a) {
  extern __shared__ __align__(16) double tsm_[];
  constexpr int NC = 32 * JC;
  const int ndp = tile_ndp(a.nd);
  double* F = tsm_;                                            // [ndp][NC]
  double* A = F + ndp * NC;                                    // [kTileRows][ndp]
  float* Af = reinterpret_cast<float*>(A + kTileRows * ndp);  // [kTileRows][ndp]
  float* Bf = Af + kTileRows * ndp;                            // [kTileRows][nb0]
  int* dw = reinterpret_cast<int*>(Bf + kTileRows * a.nb0);    // [nd]
  int* bz = dw + a.nd;                                         // [nb0]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the transposed fit, columns nsh.. NC-1 and rows nd.. ndp-1 zero
  for (int i = threadIdx.x; i < ndp * NC; i += blockDim.x) {
    const int k = i / NC, c = i - k * NC;
    F[i] = (k < a.nd && c < a.nsh) ? a.fit[(long long)c * a.nd + k] : 0.0;
  }
  for (int t = threadIdx.x; t < a.nd; t += blockDim.x) dw[t] = a.dwis[t];
  for (int t = threadIdx.x; t < a.nb0; t += blockDim.x) bz[t] = a.b0[t];
  __syncthreads();
  // gathers a tile's amplitudes into Af / Bf: cp.async, in flight while the
  // previous tile computes (rows past the last voxel are not gathered)
  auto gather = [&](long long tile) {
    for (int r = warp; r < kTileRows; r += kTileWarps) {
      const long long v = tile * kTileRows + r;
      if (v >= a.n) break;
      const float* p = a.amp + v * a.vs;
      for (int t = lane; t < a.nd; t += 32) cp_async4(Af + r * ndp + t, p + (long long)dw[t] * a.ts);
      if (a.normalise)
        for (int t = lane; t < a.nb0; t += 32) cp_async4(Bf + r * a.nb0 + t, p + (long long)bz[t] * a.ts);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const long long ntiles = (a.n + kTileRows - 1) / kTileRows;
  if ((long long)blockIdx.x < ntiles) gather(blockIdx.x);
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long v0 = tile * kTileRows;
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();  // this tile's staging visible; the previous tile's A consumed
    for (int r = warp; r < kTileRows; r += kTileWarps) {
      double* row = A + r * ndp;
      if (v0 + r >= a.n) {
        for (int t = lane; t < ndp; t += 32) row[t] = 0.0;
        continue;
      }
      double norm = 1.0;
      if (a.normalise) {
        double s = 1.0;  // get_amps' order, as above
        for (int i = 0; i < a.nb0; ++i) s += (double)Bf[r * a.nb0 + i];
        norm = (double)a.nb0 / s;
      }
      for (int t = lane; t < ndp; t += 32) row[t] = t < a.nd ? (double)Af[r * ndp + t] * norm : 0.0;
    }
    __syncthreads();  // A ready; Af / Bf free for the next tile
    if (tile + gridDim.x < ntiles) gather(tile + gridDim.x);
    double acc[kTileVox][JC];
#pragma unroll
    for (int i = 0; i < kTileVox; ++i)
#pragma unroll
      for (int j = 0; j < JC; ++j) acc[i][j] = 0.0;
    const double* Aw = A + warp * kTileVox * ndp;
#pragma unroll 2
    for (int k = 0; k < ndp; k += 2) {
      double f0[JC], f1[JC];
#pragma unroll
      for (int j = 0; j < JC; ++j) {
        f0[j] = F[k * NC + lane + 32 * j];
        f1[j] = F[(k + 1) * NC + lane + 32 * j];
      }
#pragma unroll
      for (int i = 0; i < kTileVox; ++i) {
        const double2 x = *reinterpret_cast<const double2*>(Aw + i * ndp + k);
#pragma unroll
        for (int j = 0; j < JC; ++j) acc[i][j] = fma(f1[j], x.y, fma(f0[j], x.x, acc[i][j]));
      }
    }
#pragma unroll
    for (int i = 0; i < kTileVox; ++i) {
      const long long v = v0 + warp * kTileVox + i;
      if (v >= a.n) break;
#pragma unroll
      for (int j = 0; j < JC; ++j) {
        const int c = lane + 32 * j;
        if (c < a.nsh) a.out[v * a.os + c] = (float)acc[i][j];
      }
    }
  }
}

// ---- FP64 tensor-core kernel (mma.sync m8n8k4 f64) for fits of nd <= 64
// directions and nSH <= 48 columns (lmax <= 8).  D [voxels][columns] =
// A [voxels][directions] x B [directions][columns], B = fit^T; the b=0
// normalisation scales D's rows (norm (fit a) = fit (norm a)).  The block
// has 2 x WN warps: warp (wm, wn) forms 4 m-tiles (32 voxels) x 1 n-tile (8
// columns) of the block's 64 voxels, with its B fragments for all k-steps
// held in registers for the life of the block; two blocks an SM, so that
// one block's staging overlaps the other's products.  The next tile's
// amplitudes arrive by cp.async while the current one computes: whole voxel
// rows in 16-byte pieces when the volumes are contiguous (volume stride 1,
// 16-byte aligned amplitudes), else the selected volumes one by one.  A is
// then converted to double in fragment order, [m-tile][k-step pair][lane][2],
// so that a lane's operands for two k-steps are one 16-byte load.  Fragment
// layouts (PTX ISA, mma.m8n8k4 .f64): A a0 = A[lane / 4][lane % 4]; B b0 =
// B[lane % 4][lane / 4]; C / D c_i = C[lane / 4][2 (lane % 4) + i].
constexpr int kMmaWM = 2;    // warps along the voxels
constexpr int kMmaMT = 4;    // m-tiles (8 voxels) a warp forms: 2 x 4 x 8 = 64
constexpr int kMmaNTW = 1;   // n-tiles (8 columns) a warp forms
constexpr int kMmaKSM = 16;  // k-steps (4 directions) a warp holds: nd <= 64
constexpr int kMmaMaxWarps = kMmaWM * 6;  // nSH <= 48 (lmax <= 8): at most 6 warps along the columns
constexpr int kMmaMaxRow = 256;           // longest voxel row staged whole (floats)

__host__ __device__ inline int mma_ks2(int nd) { return ((nd + 3) / 4 + 1) / 2; }
// staged floats a voxel: the whole row (contiguous volumes) or the selected ones
__host__ inline int mma_row_floats(int nd, int nb0, bool whole_rows, long long vs) {
  return whole_rows ? (int)std::max<long long>(vs, nd + nb0) : nd + nb0;
}
__host__ inline size_t mma_smem_bytes(int nd, int nb0, int row_floats) {
  return ((size_t)kTileRows * mma_ks2(nd) * 8 + kTileRows) * sizeof(double) +
         ((size_t)kTileRows * row_floats + nd + nb0) * sizeof(float);
}

__device__ __forceinline__ void dmma_m8n8k4(double& c0, double& c1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

__global__ void __launch_bounds__(kMmaMaxWarps * 32, 2) amp2sh_mma_kernel(const __grid_constant__ Amp2ShArgs a) {
  extern __shared__ __align__(16) double msm_[];
  const int ks = (a.nd + 3) / 4, ks2 = mma_ks2(a.nd);
  double* Ap = msm_;                                              // [8][ks2][32][2]
  double* nrm = Ap + kTileRows * ks2 * 8;                         // [kTileRows]
  float* S = reinterpret_cast<float*>(nrm + kTileRows);          // [kTileRows][row_floats]
  int* dw = reinterpret_cast<int*>(S + kTileRows * a.row_floats);  // [nd]
  int* bz = dw + a.nd;                                            // [nb0]
  __shared__ int max_index;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const int wm = warp % kMmaWM, wn = warp / kMmaWM;
  double b[kMmaKSM];
  {
    const int c = 8 * wn + (lane >> 2);
#pragma unroll
    for (int ks = 0; ks < kMmaKSM; ++ks) {
      const int k = 4 * ks + (lane & 3);
      b[ks] = (k < a.nd && c < a.nsh) ? __ldg(a.fit + (long long)c * a.nd + k) : 0.0;
    }
  }
  if (threadIdx.x == 0) max_index = 0;
  __syncthreads();
  for (int t = threadIdx.x; t < a.nd; t += blockDim.x) {
    dw[t] = a.dwis[t];
    atomicMax(&max_index, dw[t]);
  }
  for (int t = threadIdx.x; t < a.nb0; t += blockDim.x) {
    bz[t] = a.b0[t];
    atomicMax(&max_index, bz[t]);
  }
  __syncthreads();
  // whole rows only when every selected volume lies inside the row
  const bool whole = a.contig && max_index < a.vs;
  // staged row stride: the voxel stride for whole rows, else the selection
  const int ls = whole ? (int)a.vs : a.nd + a.nb0;
  // this lane's two conversion slots t = lane, lane + 32: the staged float it
  // reads (-1: padding) and its place in an m-tile's fragment-ordered rows
  int src[2], dst[2];
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int t = lane + 32 * j;
    src[j] = t < a.nd ? (whole ? dw[t] : t) : -1;
    dst[j] = (t >> 3) * 64 + (t & 3) * 2 + ((t >> 2) & 1);
  }
  auto gather = [&](long long tile) {
    const long long v0 = tile * kTileRows;
    const int rows = a.n - v0 < kTileRows ? (int)(a.n - v0) : kTileRows;
    if (whole) {
      // rows v0 .. v0 + rows - 1 up to the last voxel's highest selected volume
      const float* base = a.amp + v0 * a.vs;
      const int nfl = (rows - 1) * (int)a.vs + max_index + 1;
      const int nch = nfl >> 2;
      for (int c = threadIdx.x; c < nch; c += blockDim.x) cp_async16(S + 4 * c, base + 4 * c);
      for (int e = 4 * nch + threadIdx.x; e < nfl; e += blockDim.x) cp_async4(S + e, base + e);
    } else {
      for (int r = warp; r < rows; r += nwarps) {
        const float* p = a.amp + (v0 + r) * a.vs;
        for (int t = lane; t < a.nd; t += 32) cp_async4(S + r * ls + t, p + (long long)dw[t] * a.ts);
        if (a.normalise)
          for (int t = lane; t < a.nb0; t += 32) cp_async4(S + r * ls + a.nd + t, p + (long long)bz[t] * a.ts);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  const long long ntiles = (a.n + kTileRows - 1) / kTileRows;
  if ((long long)blockIdx.x < ntiles) gather(blockIdx.x);
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long v0 = tile * kTileRows;
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();  // this tile's staging visible; the previous tile's A consumed
    for (int r = warp; r < kTileRows; r += nwarps) {
      const bool live = v0 + r < a.n;
      const float* row = S + r * ls;
      double* out = Ap + (r >> 3) * ks2 * 64 + (r & 7) * 8;
#pragma unroll
      for (int j = 0; j < 2; ++j)
        if (lane + 32 * j < 8 * ks2) out[dst[j]] = (live && src[j] >= 0) ? (double)row[src[j]] : 0.0;
    }
    if (a.normalise)
      for (int r = threadIdx.x; r < kTileRows; r += blockDim.x) {
        if (v0 + r >= a.n) continue;
        // get_amps' sum, in its order: 1 + the b=0 amplitudes one by one
        double s = 1.0;
        for (int i = 0; i < a.nb0; ++i) s += (double)S[r * ls + (whole ? bz[i] : a.nd + i)];
        nrm[r] = (double)a.nb0 / s;
      }
    __syncthreads();  // A and the norms ready; the staging free for the next tile
    if (tile + gridDim.x < ntiles) gather(tile + gridDim.x);
    double acc[kMmaMT][2];
#pragma unroll
    for (int m = 0; m < kMmaMT; ++m) acc[m][0] = acc[m][1] = 0.0;
#pragma unroll
    for (int kp = 0; kp < kMmaKSM / 2; ++kp) {
      if (kp < ks2) {
        double2 x[kMmaMT];
#pragma unroll
        for (int m = 0; m < kMmaMT; ++m)
          x[m] = *reinterpret_cast<const double2*>(Ap + (((wm * kMmaMT + m) * ks2 + kp) * 32 + lane) * 2);
#pragma unroll
        for (int m = 0; m < kMmaMT; ++m) dmma_m8n8k4(acc[m][0], acc[m][1], x[m].x, b[2 * kp]);
        if (2 * kp + 1 < ks)  // an odd k-step count leaves the last pair's second step empty
#pragma unroll
          for (int m = 0; m < kMmaMT; ++m) dmma_m8n8k4(acc[m][0], acc[m][1], x[m].y, b[2 * kp + 1]);
      }
    }
    const int c = 8 * wn + 2 * (lane & 3);
#pragma unroll
    for (int m = 0; m < kMmaMT; ++m) {
      const int r = (wm * kMmaMT + m) * 8 + (lane >> 2);
      const long long v = v0 + r;
      if (v < a.n) {
        const double f = a.normalise ? nrm[r] : 1.0;
        if (c < a.nsh) a.out[v * a.os + c] = (float)(acc[m][0] * f);
        if (c + 1 < a.nsh) a.out[v * a.os + c + 1] = (float)(acc[m][1] * f);
      }
    }
  }
}

template <int JC>
cudaError_t launch_tile(const Amp2ShArgs& a, size_t smem, int nsm, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(amp2sh_tile_kernel<JC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amp2sh_tile_kernel<JC>, kTileWarps * 32, smem);
  if (e != cudaSuccess) return e;
  const long long tiles = (a.n + kTileRows - 1) / kTileRows;
  const long long grid = std::max<long long>(1, std::min<long long>(tiles, (long long)nsm * std::max(1, per_sm)));
  amp2sh_tile_kernel<JC><<<(unsigned)grid, kTileWarps * 32, smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

extern "C" int csd_amp2sh(const float* amp, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                          const double* fit, int nsh, const int* dwis, int nd, const int* bzeros, int nb0,
                          int normalise, float* sh_out, int64_t out_stride, void* stream) {
  if (n_voxels < 0 || (n_voxels > 0 && (!amp || !sh_out)) || !fit || !dwis || nd < 1 || nd > kA2sMaxDirs || nsh < 1 ||
      out_stride < nsh || nb0 < 0 || (nb0 && !bzeros) || (normalise && nb0 == 0))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_amp2sh: invalid argument (normalising needs b=0 volumes)");
  if (n_voxels == 0) return CSD_OK;
  Amp2ShArgs a{};
  a.amp = amp;
  a.n = n_voxels;
  a.vs = voxel_stride;
  a.ts = volume_stride;
  a.fit = fit;
  a.dwis = dwis;
  a.b0 = bzeros;
  a.nd = nd;
  a.nb0 = nb0;
  a.nsh = nsh;
  a.normalise = normalise;
  a.out = sh_out;
  a.os = out_stride;
  int dev = 0, nsm = 0, smem_max = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_amp2sh: ") + cudaGetErrorString(e));
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int jc = (nsh + 31) / 32;
  const bool mma_ok = nd <= 4 * kMmaKSM && nsh <= 8 * kMmaNTW * (kMmaMaxWarps / kMmaWM) &&
                      mma_smem_bytes(nd, nb0, mma_row_floats(nd, nb0, false, 0)) <= (size_t)smem_max / 2;
  // the whole fit in shared memory with room for two blocks an SM
  const bool tile_ok = jc <= 3 && tile_smem_bytes(nd, nb0, jc) <= (size_t)smem_max / 2;
  const int want = csdb200::g_amp2sh_kind;
  const int kind = want == 1 ? 1 : (want == 2 && tile_ok) ? 2 : (want == 3 && mma_ok) ? 3 : mma_ok ? 3 : tile_ok ? 2 : 1;
  if (kind == 3) {
    // whole voxel rows staged when the volumes are contiguous and each tile's
    // first row is 16-byte aligned (tiles start 64 rows apart)
    a.contig = volume_stride == 1 && voxel_stride >= 1 && voxel_stride <= kMmaMaxRow &&
               (reinterpret_cast<uintptr_t>(amp) & 15) == 0;
    a.row_floats = mma_row_floats(nd, nb0, a.contig, voxel_stride);
    size_t smem = mma_smem_bytes(nd, nb0, a.row_floats);
    if (smem > (size_t)smem_max / 2) {  // two blocks an SM or the selected volumes only
      a.contig = 0;
      a.row_floats = mma_row_floats(nd, nb0, false, voxel_stride);
      smem = mma_smem_bytes(nd, nb0, a.row_floats);
    }
    const int wn = ((nsh + 7) / 8 + kMmaNTW - 1) / kMmaNTW;
    const int threads = 32 * kMmaWM * wn;
    int per_sm = 0;
    e = cudaFuncSetAttribute(amp2sh_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amp2sh_mma_kernel, threads, smem);
    if (e == cudaSuccess) {
      const long long tiles = (n_voxels + kTileRows - 1) / kTileRows;
      const long long grid = std::max<long long>(1, std::min<long long>(tiles, (long long)nsm * std::max(1, per_sm)));
      amp2sh_mma_kernel<<<(unsigned)grid, threads, smem, st>>>(a);
      e = cudaGetLastError();
    }
  } else if (kind == 2) {
    const size_t smem = tile_smem_bytes(nd, nb0, jc);
    e = jc == 1 ? launch_tile<1>(a, smem, nsm, st) : jc == 2 ? launch_tile<2>(a, smem, nsm, st)
                                                      : launch_tile<3>(a, smem, nsm, st);
  } else {
    const size_t smem = (size_t)kA2sRows * (nd + 1) * sizeof(double);
    e = cudaFuncSetAttribute(amp2sh_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) {
      const long long tiles = (n_voxels + kA2sRows - 1) / kA2sRows;
      amp2sh_kernel<<<(unsigned)std::max<long long>(1, std::min<long long>(tiles, (long long)nsm * 8)), kA2sThreads,
                      smem, st>>>(a);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_amp2sh: ") + cudaGetErrorString(e));
  return CSD_OK;
}

// ---- amp2sh -rician (amp2sh.cpp:129-150, 180-197): the fit reweighted for
// the Rician noise bias.  Per voxel, from c = fit a: up to 20 rounds of
//   ap = SH2amp c, clamped at 0; t = (ap / noise)^2.25;
//   w = ((t + 1.7) / (t + 1.12))^2; diff = a - noise (t + 1.65)^(1 / 2.25);
//   stop when sum diff^2 / sum a^2 < 1e-8; else ap += diff and
//   c = (H^T H)^-1 H^T ap with H = diag(w) SH2amp (Cholesky, as LLT there).
// A warp a voxel, in FP64; per warp in shared memory: a, ap, w [nd], c, s
// [nsh] and the packed lower triangle of H^T H.
namespace {

constexpr int kRicWarps = 4;
constexpr int kRicRounds = 20;
constexpr double kRicianPower = 2.25;

__host__ __device__ inline size_t ric_warp_doubles(int nd, int nsh) {
  return 3 * (size_t)nd + 2 * (size_t)nsh + (size_t)nsh * (nsh + 1) / 2;
}

struct RicianArgs {
  Amp2ShArgs a;
  const double* sh2amp;  // [nd][nsh]
  const float* noise;    // [n] (noise[v * noise_stride])
  long long noise_stride;
};

__device__ __forceinline__ double ric_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kRicWarps * 32) amp2sh_rician_kernel(const __grid_constant__ RicianArgs ra) {
  extern __shared__ __align__(16) double rsm_[];
  const Amp2ShArgs& a = ra.a;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nd = a.nd, nsh = a.nsh;
  double* av = rsm_ + warp * ric_warp_doubles(nd, nsh);
  double* ap = av + nd;
  double* w = ap + nd;
  double* c = w + nd;
  double* s = c + nsh;
  double* Q = s + nsh;  // packed lower: Q[i (i + 1) / 2 + j]
  const long long gw = (long long)blockIdx.x * kRicWarps + warp, nw = (long long)gridDim.x * kRicWarps;
  for (long long v = gw; v < a.n; v += nw) {
    const float* p = a.amp + v * a.vs;
    double norm = 1.0;
    if (a.normalise) {
      double t = 1.0;  // get_amps' order
      for (int i = 0; i < a.nb0; ++i) t += (double)p[(long long)a.b0[i] * a.ts];
      norm = (double)a.nb0 / t;
    }
    for (int n = lane; n < nd; n += 32) av[n] = (double)p[(long long)a.dwis[n] * a.ts] * norm;
    __syncwarp();
    for (int j = lane; j < nsh; j += 32) {
      const double* f = a.fit + (long long)j * nd;
      double t = 0.0;
      for (int n = 0; n < nd; ++n) t = fma(f[n], av[n], t);
      c[j] = t;
    }
    __syncwarp();
    const double noise = (double)ra.noise[v * ra.noise_stride];
    for (int round = 0; round < kRicRounds; ++round) {
      // get_rician_bias: ap, w, the convergence test, ap += diff
      double nd2 = 0.0, na2 = 0.0;
      for (int n = lane; n < nd; n += 32) {
        const double* h = ra.sh2amp + (long long)n * nsh;
        double t = 0.0;
        for (int j = 0; j < nsh; ++j) t = fma(h[j], c[j], t);
        t = fmax(t, 0.0);
        const double tt = pow(t / noise, kRicianPower);
        const double q = (tt + 1.7) / (tt + 1.12);
        w[n] = q * q;
        const double diff = av[n] - noise * pow(tt + 1.65, 1.0 / kRicianPower);
        nd2 = fma(diff, diff, nd2);
        na2 = fma(av[n], av[n], na2);
        ap[n] = t + diff;
      }
      nd2 = ric_warp_sum(nd2);
      na2 = ric_warp_sum(na2);
      __syncwarp();
      if (nd2 / na2 < 1.0e-8) break;
      // s = H^T ap, Q = H^T H (lower), H = diag(w) SH2amp
      for (int j = lane; j < nsh; j += 32) {
        double t = 0.0;
        for (int n = 0; n < nd; ++n) t = fma(ra.sh2amp[(long long)n * nsh + j] * w[n], ap[n], t);
        s[j] = t;
      }
      const int nq = nsh * (nsh + 1) / 2;
      for (int e = lane; e < nq; e += 32) {
        int i = (int)((sqrt(8.0 * e + 1.0) - 1.0) * 0.5);
        while (i * (i + 1) / 2 > e) --i;
        while ((i + 1) * (i + 2) / 2 <= e) ++i;
        const int j = e - i * (i + 1) / 2;
        double t = 0.0;
        for (int n = 0; n < nd; ++n) {
          const double wn = w[n];
          t = fma(ra.sh2amp[(long long)n * nsh + i] * wn, ra.sh2amp[(long long)n * nsh + j] * wn, t);
        }
        Q[e] = t;
      }
      __syncwarp();
      // Cholesky in place (left-looking by columns; lanes over the rows)
      for (int k = 0; k < nsh; ++k) {
        const int kk = k * (k + 1) / 2;
        double d = 0.0;
        for (int m = lane; m < k; m += 32) d = fma(Q[kk + m], Q[kk + m], d);
        d = ric_warp_sum(d);
        const double dk = sqrt(Q[kk + k] - d);
        __syncwarp();
        for (int i = k + 1 + lane; i < nsh; i += 32) {
          const int ii = i * (i + 1) / 2;
          double t = Q[ii + k];
          for (int m = 0; m < k; ++m) t -= Q[ii + m] * Q[kk + m];
          Q[ii + k] = t / dk;
        }
        __syncwarp();
        if (lane == 0) Q[kk + k] = dk;
        __syncwarp();
      }
      // c = L^-T L^-1 s (column-oriented substitutions)
      for (int k = 0; k < nsh; ++k) {
        const double zk = s[k] / Q[k * (k + 1) / 2 + k];
        __syncwarp();
        for (int i = k + 1 + lane; i < nsh; i += 32) s[i] -= Q[i * (i + 1) / 2 + k] * zk;
        if (lane == 0) s[k] = zk;
        __syncwarp();
      }
      for (int k = nsh - 1; k >= 0; --k) {
        const int kk = k * (k + 1) / 2;
        const double ck = s[k] / Q[kk + k];
        __syncwarp();
        for (int i = lane; i < k; i += 32) s[i] -= Q[kk + i] * ck;
        if (lane == 0) s[k] = ck;
        __syncwarp();
      }
      for (int j = lane; j < nsh; j += 32) c[j] = s[j];
      __syncwarp();
    }
    for (int j = lane; j < nsh; j += 32) a.out[v * a.os + j] = (float)c[j];
    __syncwarp();
  }
}

}  // namespace

extern "C" int csd_amp2sh_rician(const float* amp, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                                 const double* fit, const double* sh2amp, int nsh, const int* dwis, int nd,
                                 const int* bzeros, int nb0, int normalise, const float* noise, int64_t noise_stride,
                                 float* sh_out, int64_t out_stride, void* stream) {
  if (n_voxels < 0 || (n_voxels > 0 && (!amp || !sh_out || !noise)) || !fit || !sh2amp || !dwis || nd < 1 ||
      nd > kA2sMaxDirs || nsh < 1 || nsh > 153 || out_stride < nsh || nb0 < 0 || (nb0 && !bzeros) ||
      (normalise && nb0 == 0))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_amp2sh_rician: invalid argument");
  if (n_voxels == 0) return CSD_OK;
  RicianArgs ra{};
  Amp2ShArgs& a = ra.a;
  a.amp = amp;
  a.n = n_voxels;
  a.vs = voxel_stride;
  a.ts = volume_stride;
  a.fit = fit;
  a.dwis = dwis;
  a.b0 = bzeros;
  a.nd = nd;
  a.nb0 = nb0;
  a.nsh = nsh;
  a.normalise = normalise;
  a.out = sh_out;
  a.os = out_stride;
  ra.sh2amp = sh2amp;
  ra.noise = noise;
  ra.noise_stride = noise_stride;
  int dev = 0, nsm = 0, smem_max = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const size_t smem = kRicWarps * ric_warp_doubles(nd, nsh) * sizeof(double);
  if (e == cudaSuccess && smem > (size_t)smem_max)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_amp2sh_rician: problem too large for shared memory");
  if (e == cudaSuccess) e = cudaFuncSetAttribute(amp2sh_rician_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per_sm = 0;
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, amp2sh_rician_kernel, kRicWarps * 32, smem);
  if (e == cudaSuccess) {
    const long long blocks = std::max<long long>(
        1, std::min<long long>((n_voxels + kRicWarps - 1) / kRicWarps, (long long)nsm * std::max(1, per_sm)));
    amp2sh_rician_kernel<<<(unsigned)blocks, kRicWarps * 32, smem, static_cast<cudaStream_t>(stream)>>>(ra);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_amp2sh_rician: ") + cudaGetErrorString(e));
  return CSD_OK;
}
