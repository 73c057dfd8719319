// amp2response on the GPU: the accumulation of the response-function fit
// over single-fibre voxels (MRtrix3 cmd/amp2response.cpp:152-190).  For every
// voxel of the mask and every volume i of a shell, with d_i the volume's
// unit direction and f the voxel's fibre direction (normalised), the
// elevation of d_i in the fibre's frame, folded into [0, pi/2]
// (amp2response.cpp:159-173: only |f . d_i| matters, whatever the two
// random in-plane axes), gives the zonal basis row T_i = [P_l0(cos el)]
// (l = 0, 2, .., lmax; core/math/ZSH.h:66-77); M += T^T T and b += T^T a with
// a_i the voxel's amplitude of volume i.  FP64; a thread per (voxel, volume)
// pair, reduced over the block, then added into M (lower triangle) and b.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/csd_b200.h"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu
}

namespace {

constexpr int kArMaxLmax = 12;
constexpr int kArMaxZ = kArMaxLmax / 2 + 1;                  // 7 zonal terms
constexpr int kArAcc = kArMaxZ * (kArMaxZ + 1) / 2 + kArMaxZ;  // lower M + b
constexpr int kArThreads = 256;

struct ArArgs {
  const float* amp;
  long long n, vs, ts;
  const float* fdir;
  long long ds, dcs;
  const uint8_t* mask;
  const double* dirs;  // [nd][3]
  const int* vols;     // [nd]
  int nd, lmax, nz;
  double* M;  // [nz][nz], lower triangle accumulated
  double* b;  // [nz]
};

__global__ void __launch_bounds__(kArThreads) amp2response_kernel(const __grid_constant__ ArArgs a) {
  double acc[kArAcc];
#pragma unroll
  for (int k = 0; k < kArAcc; ++k) acc[k] = 0.0;
  const long long total = a.n * a.nd;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long v = e / a.nd;
    const int i = (int)(e - v * a.nd);
    if (a.mask && !a.mask[v]) continue;
    const float* fd = a.fdir + v * a.ds;
    double fx = fd[0], fy = fd[a.dcs], fz = fd[2 * a.dcs];
    const double fn = sqrt(fx * fx + fy * fy + fz * fz);
    fx /= fn;
    fy /= fn;
    fz /= fn;
    const double* d = a.dirs + 3 * (long long)i;
    const double z = (fx * d[0] + fy * d[1] + fz * d[2]) / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double el = acos(fmin(fmax(z, -1.0), 1.0));
    if (el > 1.5707963267948966) el = 3.141592653589793 - el;
    if (z != z) el = z;  // an undefined direction stays undefined (NaN)
    const double x = cos(el);
    // normalised Legendre P_l0 (core/math/legendre.h:101-123 with m = 0)
    double T[kArMaxZ];
    double p0 = 0.282094791773878, p1 = 0.0;
    T[0] = p0;
#pragma unroll
    for (int r = 1; r < kArMaxZ; ++r) T[r] = 0.0;
    double f = sqrt(3.0);
    p1 = x * f * p0;
#pragma unroll
    for (int l = 2; l <= kArMaxLmax; ++l) {
      if (l <= a.lmax) {
        double pl = x * p1 - p0 / f;
        f = sqrt((4.0 * l * l - 1.0) / ((double)l * l));
        pl *= f;
        p0 = p1;
        p1 = pl;
        if (!(l & 1)) T[l >> 1] = pl;
      }
    }
    const double av = (double)a.amp[v * a.vs + (long long)a.vols[i] * a.ts];
    int k = 0;
#pragma unroll
    for (int r = 0; r < kArMaxZ; ++r)
#pragma unroll
      for (int c = 0; c <= r; ++c, ++k)
        if (r < a.nz) acc[k] = fma(T[r], T[c], acc[k]);
#pragma unroll
    for (int r = 0; r < kArMaxZ; ++r)
      if (r < a.nz) acc[k + r] = fma(T[r], av, acc[k + r]);
  }
  // block reduction, then one atomic add per term
  __shared__ double red[kArThreads / 32][kArAcc];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kArAcc; ++k) {
    double s = acc[k];
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp][k] = s;
  }
  __syncthreads();
  if (threadIdx.x < kArAcc) {
    double s = 0.0;
    for (int w = 0; w < kArThreads / 32; ++w) s += red[w][threadIdx.x];
    const int k = threadIdx.x;
    const int nlow = kArMaxZ * (kArMaxZ + 1) / 2;
    if (k < nlow) {
      int r = 0;
      while ((r + 1) * (r + 2) / 2 <= k) ++r;
      const int c = k - r * (r + 1) / 2;
      if (r < a.nz) atomicAdd(&a.M[r * a.nz + c], s);
    } else if (k - nlow < a.nz) {
      atomicAdd(&a.b[k - nlow], s);
    }
  }
}

}  // namespace

extern "C" int csd_amp2response_accumulate(const float* amp, int64_t n_voxels, int64_t voxel_stride,
                                           int64_t volume_stride, const float* fibre_dir, int64_t dir_stride,
                                           int64_t dir_comp_stride, const uint8_t* mask, const double* dirs,
                                           int n_dirs, const int* volumes, int lmax, double* M, double* b,
                                           void* stream) {
  if (n_voxels < 0 || (n_voxels > 0 && (!amp || !fibre_dir)) || !dirs || !volumes || n_dirs < 1 || lmax < 0 ||
      lmax > kArMaxLmax || (lmax & 1) || !M || !b)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_amp2response_accumulate: invalid argument (lmax even, <= 12)");
  if (n_voxels == 0) return CSD_OK;
  ArArgs a{};
  a.amp = amp;
  a.n = n_voxels;
  a.vs = voxel_stride;
  a.ts = volume_stride;
  a.fdir = fibre_dir;
  a.ds = dir_stride;
  a.dcs = dir_comp_stride;
  a.mask = mask;
  a.dirs = dirs;
  a.vols = volumes;
  a.nd = n_dirs;
  a.lmax = lmax;
  a.nz = lmax / 2 + 1;
  a.M = M;
  a.b = b;
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) {
    const long long total = n_voxels * n_dirs;
    const long long blocks = std::max<long long>(1, std::min<long long>((total + kArThreads - 1) / kArThreads,
                                                                         (long long)nsm * 8));
    amp2response_kernel<<<(unsigned)blocks, kArThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_amp2response_accumulate: ") + cudaGetErrorString(e));
  return CSD_OK;
}
