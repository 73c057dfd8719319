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
        double s = 0.0;
        for (int i = lane; i < a.nb0; i += 32) s += (double)p[(long long)a.b0[i] * a.ts];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        norm = (double)a.nb0 / (1.0 + s);
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
        double s = 0.0;
        for (int i = lane; i < a.nb0; i += 32) s += (double)Bf[r * a.nb0 + i];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        norm = (double)a.nb0 / (1.0 + s);
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
  if (jc <= 3 && tile_smem_bytes(nd, nb0, jc) <= (size_t)smem_max / 2) {
    // the whole fit in shared memory with room for two blocks an SM
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
