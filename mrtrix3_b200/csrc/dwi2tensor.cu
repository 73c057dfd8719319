// dwi2tensor on the GPU with the tensor2metric values dwi2response needs
// (MRtrix3 cmd/dwi2tensor.cpp:106-135, src/dwi/tensor.h:30-56, 95-104,
// cmd/tensor2metric.cpp:156-247).  A thread per voxel, FP64:
//   S clamped below at 1e-6 of the voxel's largest value, y = ln S, weights w
//   = S (1 with -ols); for it = 0..iter: p = (B^T W^2 B)^-1 B^T W^2 y
//   (Cholesky of the 7 x 7 normal matrix), then w = exp(B p) unless last;
//   B = -grad2bmatrix: rows [-b gx^2, -b gy^2, -b gz^2, -2b gx gy, -2b gx gz,
//   -2b gy gz, 1].  Outputs the tensor [Dxx Dyy Dzz Dxy Dxz Dyz], b0 =
//   exp(p6), FA (tensor2FA) and the principal eigenvector modulated by FA
//   (tensor2metric -vector's default; cyclic Jacobi rotations on the 3 x 3
//   tensor instead of Eigen's SelfAdjointEigenSolver: the same vector up to
//   its sign, which is arbitrary there too).
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

constexpr int kDtThreads = 128;

struct DtArgs {
  const float* dwi;
  long long n, vs, ts;
  const double* bmat;  // [nvol][7]
  int nvol, iter, ols;
  const uint8_t* mask;
  float* dt;
  long long dts;
  float* b0;
  float* fa;
  float* vec;
};

__device__ __forceinline__ int tri(int i, int j) { return i * (i + 1) / 2 + j; }

__global__ void __launch_bounds__(kDtThreads) dwi2tensor_kernel(const __grid_constant__ DtArgs a) {
  for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < a.n; v += (long long)gridDim.x * blockDim.x) {
    float* dto = a.dt + v * a.dts;
    if (a.mask && !a.mask[v]) {
      for (int j = 0; j < 6; ++j) dto[j] = 0.f;
      if (a.b0) a.b0[v] = 0.f;
      if (a.fa) a.fa[v] = 0.f;
      if (a.vec) a.vec[3 * v] = a.vec[3 * v + 1] = a.vec[3 * v + 2] = 0.f;
      continue;
    }
    const float* s = a.dwi + v * a.vs;
    double smax = -INFINITY;
    for (int i = 0; i < a.nvol; ++i) smax = fmax(smax, (double)s[(long long)i * a.ts]);
    const double small = 1.0e-6 * smax;
    double p[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) p[j] = 0.0;
    for (int it = 0; it <= a.iter; ++it) {
      double A[28], r[7];
#pragma unroll
      for (int k = 0; k < 28; ++k) A[k] = 0.0;
#pragma unroll
      for (int k = 0; k < 7; ++k) r[k] = 0.0;
      for (int i = 0; i < a.nvol; ++i) {
        const double* bi = a.bmat + 7 * (long long)i;
        double si = (double)s[(long long)i * a.ts];
        if (si < small) si = small;
        const double y = log(si);
        double w;
        if (it == 0) {
          w = a.ols ? 1.0 : si;
        } else {
          double e = 0.0;
#pragma unroll
          for (int j = 0; j < 7; ++j) e = fma(__ldg(bi + j), p[j], e);
          w = exp(e);
        }
        const double w2 = w * w;
        double bw[7];
#pragma unroll
        for (int j = 0; j < 7; ++j) bw[j] = __ldg(bi + j) * w2;
#pragma unroll
        for (int j = 0; j < 7; ++j) {
#pragma unroll
          for (int k = 0; k <= j; ++k) A[tri(j, k)] = fma(bw[j], __ldg(bi + k), A[tri(j, k)]);
          r[j] = fma(bw[j], y, r[j]);
        }
      }
      // Cholesky (packed lower) and the two substitutions
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        double d = A[tri(j, j)];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= A[tri(j, k)] * A[tri(j, k)];
        d = sqrt(d);
        A[tri(j, j)] = d;
#pragma unroll
        for (int i = j + 1; i < 7; ++i) {
          double t = A[tri(i, j)];
#pragma unroll
          for (int k = 0; k < j; ++k) t -= A[tri(i, k)] * A[tri(j, k)];
          A[tri(i, j)] = t / d;
        }
      }
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        double t = r[i];
#pragma unroll
        for (int k = 0; k < i; ++k) t -= A[tri(i, k)] * r[k];
        r[i] = t / A[tri(i, i)];
      }
#pragma unroll
      for (int i = 6; i >= 0; --i) {
        double t = r[i];
#pragma unroll
        for (int k = i + 1; k < 7; ++k) t -= A[tri(k, i)] * r[k];
        r[i] = t / A[tri(i, i)];
      }
#pragma unroll
      for (int j = 0; j < 7; ++j) p[j] = r[j];
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) dto[j] = (float)p[j];
    if (a.b0) a.b0[v] = (float)exp(p[6]);
    // tensor2FA (tensor.h:95-104)
    const double tr = (p[0] + p[1] + p[2]) / 3.0;
    const double d0 = p[0] - tr, d1 = p[1] - tr, d2 = p[2] - tr;
    const double off = p[3] * p[3] + p[4] * p[4] + p[5] * p[5];
    const double nrm = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] + 2.0 * off;
    const double fa = nrm != 0.0 ? sqrt(1.5 * (d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * off) / nrm) : 0.0;
    if (a.fa) a.fa[v] = (float)fa;
    if (a.vec) {
      // cyclic Jacobi on M = [[Dxx Dxy Dxz] [Dxy Dyy Dyz] [Dxz Dyz Dzz]]
      double m[3][3] = {{p[0], p[3], p[4]}, {p[3], p[1], p[5]}, {p[4], p[5], p[2]}};
      double V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      for (int sweep = 0; sweep < 32; ++sweep) {
        const double o = fabs(m[0][1]) + fabs(m[0][2]) + fabs(m[1][2]);
        const double dsum = fabs(m[0][0]) + fabs(m[1][1]) + fabs(m[2][2]);
        if (!(o > 1e-300) || o <= 1e-18 * dsum) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
          const int P = pq == 2 ? 1 : 0, Q = pq == 0 ? 1 : 2;
          if (m[P][Q] == 0.0) continue;
          const double theta = (m[Q][Q] - m[P][P]) / (2.0 * m[P][Q]);
          const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
          const double c = 1.0 / sqrt(t * t + 1.0), sn = t * c;
#pragma unroll
          for (int k = 0; k < 3; ++k) {  // M <- J^T M J on the columns, then the rows
            const double mkp = m[k][P], mkq = m[k][Q];
            m[k][P] = c * mkp - sn * mkq;
            m[k][Q] = sn * mkp + c * mkq;
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const double mpk = m[P][k], mqk = m[Q][k];
            m[P][k] = c * mpk - sn * mqk;
            m[Q][k] = sn * mpk + c * mqk;
          }
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const double vkp = V[k][P], vkq = V[k][Q];
            V[k][P] = c * vkp - sn * vkq;
            V[k][Q] = sn * vkp + c * vkq;
          }
        }
      }
      int imax = 0;
      if (m[1][1] > m[imax][imax]) imax = 1;
      if (m[2][2] > m[imax][imax]) imax = 2;
      a.vec[3 * v] = (float)(V[0][imax] * fa);
      a.vec[3 * v + 1] = (float)(V[1][imax] * fa);
      a.vec[3 * v + 2] = (float)(V[2][imax] * fa);
    }
  }
}

}  // namespace

extern "C" int csd_dwi2tensor(const float* dwi, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                              const double* bmat, int n_volumes, const uint8_t* mask, int iter, int ols, float* dt,
                              int64_t dt_stride, float* b0, float* fa, float* vec, void* stream) {
  if (n_voxels < 0 || (n_voxels > 0 && (!dwi || !dt)) || !bmat || n_volumes < 7 || iter < 0 || iter > 10 ||
      dt_stride < 6)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_dwi2tensor: invalid argument");
  if (n_voxels == 0) return CSD_OK;
  DtArgs a{dwi, n_voxels, voxel_stride, volume_stride, bmat, n_volumes, iter, ols, mask, dt, dt_stride, b0, fa, vec};
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) {
    const long long blocks =
        std::max<long long>(1, std::min<long long>((n_voxels + kDtThreads - 1) / kDtThreads, (long long)nsm * 16));
    dwi2tensor_kernel<<<(unsigned)blocks, kDtThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_dwi2tensor: ") + cudaGetErrorString(e));
  return CSD_OK;
}
