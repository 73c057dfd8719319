// sh2peaks on the GPU: the peaks of each voxel's spherical-harmonic function
// (MRtrix3 cmd/sh2peaks.cpp:99-303 with core/math/SH.h:515-650).
//
// A warp takes a voxel: its coefficients go to shared memory, the lanes run
// the Newton searches of SH::get_peak from the seed directions (in FP32, as
// the reference: at most 50 steps, steps capped at MAX_DIR_CHANGE = 0.2 rad,
// converged below ANGLE_TOLERANCE = 1e-4), one step per lane per round, a
// lane taking the next seed as soon as its search ends; then the seeds are walked
// in order, drops a peak within |cos| > 0.99 of an earlier kept one or below
// the threshold, and either keeps the largest peaks or, per target
// direction, the peak of largest |cos| with it.  Output: [voxel][3 npeaks]
// amplitude-scaled directions, NaN where there is no peak (and for masked,
// non-finite or all-isotropic voxels, as check_input does).
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

constexpr int kPkMaxSeeds = 256;
constexpr int kPkMaxPeaks = 16;
constexpr int kPkWarps = 4;

struct PeakArgs {
  const float* sh;           // [n][stride]
  long long n, stride;
  const uint8_t* mask;       // [n] or NULL
  const float* vtargets;     // [n][3 npeaks] per-voxel targets, or NULL
  float* out;                // [n][3 npeaks]
  int n_seeds, npeaks, n_targets;
  float threshold;
  float seeds[kPkMaxSeeds][3];      // unit vectors (Direction(phi, theta) of sh2peaks.cpp:104)
  float targets[kPkMaxPeaks][3];    // global targets (-direction), normalised
  float plm_k[13];                  // Legendre starting-value constants K_m, m <= 12
};

// Starting values of the Legendre recursion: P_mm = K_m sin^m(el), with
// K_m = sqrt(1 / 4 pi) sqrt((2m+1) prod_{j<=m} (2j-1) / 2j), the closed form
// of legendre.h:65-68's helper product (which the reference evaluates per
// call); K_m is computed once on the host in double and passed in.
static void plm_start_table(float* k, int lmax) {
  for (int m = 0; m <= lmax; ++m) {
    double h = 1.0;
    for (int j = 1; j <= m; ++j) h *= (2.0 * j - 1.0) / (2.0 * j);
    k[m] = (float)(0.282094791773878 * std::sqrt((2.0 * m + 1.0) * h));
  }
  k[0] = 0.282094791773878f;
}

// Normalised associated Legendre functions of order m at cos / sin of the
// elevation (core/math/legendre.h:125-153), in float.
template <int L>
__device__ __forceinline__ void plm_sph(float* a, int m, float x, float s, const float* kk) {
  const float s2 = s * s;
  if (m && s2 == 0.f) {
    for (int n = m; n <= L; ++n) a[n] = 0.f;
    return;
  }
  float v = kk[0];
  if (m) {
    float sp = 1.f;
    for (int j = 0; j < m; ++j) sp *= s;
    v = kk[m] * fabsf(sp);
  }
  if (m & 1) v = -v;
  a[m] = v;
  if (L == m) return;
  float f = sqrtf((float)(2 * m + 3));
  a[m + 1] = x * f * a[m];
  for (int n = m + 2; n <= L; ++n) {
    a[n] = x * a[n - 1] - a[n - 2] / f;
    f = sqrtf((float)(4 * n * n - 1) / (float)(n * n - m * m));
    a[n] *= f;
  }
}

__device__ __forceinline__ int shi(int l, int m) { return l * (l + 1) / 2 + m; }
__device__ __forceinline__ int mpos(int l, int m) { return l * l / 4 + m; }

// SH::derivatives (SH.h:569-650), at the elevation / azimuth given by
// their cosines and sines; cos(m az), sin(m az) by the angle-addition
// recurrence instead of one sincos per order.
template <int L>
__device__ void sh_derivatives(const float* sh, float cel, float sel, float caz1, float saz1, float& amp,
                               float& d_el, float& d_az, float& d2_el, float& d2_elaz, float& d2_az,
                               const float* kk) {
  const bool atpole = sel < 1e-4f;
  float AL[(L / 2 + 1) * (L / 2 + 1)];
  float buf[L + 1];
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    plm_sph<L>(buf, m, cel, sel, kk);
#pragma unroll
    for (int l = (m & 1) ? m + 1 : m; l <= L; l += 2) AL[mpos(l, m)] = buf[l];
  }
  d_el = d_az = d2_el = d2_elaz = d2_az = 0.f;
  amp = sh[0] * AL[0];
#pragma unroll
  for (int l = 2; l <= L; l += 2) {
    const float v = sh[shi(l, 0)];
    amp += v * AL[mpos(l, 0)];
    d_el += v * sqrtf((float)(l * (l + 1))) * AL[mpos(l, 1)];
    d2_el += v * (sqrtf((float)(l * (l + 1) * (l - 1) * (l + 2))) * AL[mpos(l, 2)] - l * (l + 1) * AL[mpos(l, 0)]) / 2.f;
  }
  float cm = 1.f, sm = 0.f;
#pragma unroll
  for (int m = 1; m <= L; ++m) {
    const float c2 = cm * caz1 - sm * saz1;
    sm = sm * caz1 + cm * saz1;
    cm = c2;
    const float caz = 1.41421356237309505f * cm, saz = 1.41421356237309505f * sm;
#pragma unroll
    for (int l = (m & 1) ? m + 1 : m; l <= L; l += 2) {
      const float vp = sh[shi(l, m)], vm = sh[shi(l, -m)];
      const float pc = vp * caz + vm * saz, ps = vm * caz - vp * saz;
      amp += pc * AL[mpos(l, m)];
      float tmp = sqrtf((float)((l + m) * (l - m + 1))) * AL[mpos(l, m - 1)];
      if (l > m) tmp -= sqrtf((float)((l - m) * (l + m + 1))) * AL[mpos(l, m + 1)];
      tmp /= -2.f;
      d_el += pc * tmp;
      float tmp2 = -(float)((l + m) * (l - m + 1) + (l - m) * (l + m + 1)) * AL[mpos(l, m)];
      if (m == 1)
        tmp2 -= sqrtf((float)((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2))) * AL[mpos(l, 1)];
      else
        tmp2 += sqrtf((float)((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2))) * AL[mpos(l, m - 2)];
      if (l > m + 1) tmp2 += sqrtf((float)((l - m) * (l + m + 1) * (l - m - 1) * (l + m + 2))) * AL[mpos(l, m + 2)];
      tmp2 /= 4.f;
      d2_el += pc * tmp2;
      if (atpole) {
        d_az += ps * tmp;
      } else {
        d2_elaz += m * ps * tmp;
        d_az += m * ps * AL[mpos(l, m)];
        d2_az -= pc * m * m * AL[mpos(l, m)];
      }
    }
  }
  if (!atpole) {
    d_az /= sel;
    d2_elaz /= sel;
    d2_az /= sel * sel;
  }
}

// One step of SH::get_peak's Newton search (SH.h:517-553) from the unit
// vector v: amp receives the amplitude at v, v moves by the step; true when
// the step is below ANGLE_TOLERANCE (1e-4 rad), i.e. the search has ended
// with amp.  get_peak is at most 50 of these.
template <int L>
__device__ __forceinline__ bool peak_step(const float* sh, float& v0, float& v1, float& v2, const float* kk,
                                          float& amp) {
  // az = atan2(v1, v0), el = atan2(hypot(v0, v1), v2) of the unit vector
  // v, through their cosines and sines (atan2(0, 0) = 0 at the poles)
  const float h = hypotf(v0, v1);
  const float ce = v2, se = h;
  const float ca = h > 0.f ? v0 / h : (v0 < 0.f ? -1.f : 1.f), sa = h > 0.f ? v1 / h : 0.f;
  float dSH_del, dSH_daz, d2_del2, d2_deldaz, d2_daz2;
  sh_derivatives<L>(sh, ce, se, ca, sa, amp, dSH_del, dSH_daz, d2_del2, d2_deldaz, d2_daz2, kk);
  float del = sqrtf(dSH_del * dSH_del + dSH_daz * dSH_daz);
  float daz = 0.f;
  if (del != 0.f) {
    daz = dSH_daz / del;
    del = dSH_del / del;
  }
  const float dSH_dt = daz * dSH_daz + del * dSH_del;
  const float d2SH_dt2 = daz * daz * d2_daz2 + 2.f * daz * del * d2_deldaz + del * del * d2_del2;
  float dt = d2SH_dt2 != 0.f ? (-dSH_dt / d2SH_dt2) : 0.2f;
  if (dt < 0.f) dt = -dt;
  if (dt > 0.2f) dt = 0.2f;
  del *= dt;
  daz *= dt;
  v0 += del * ca * ce - daz * sa;
  v1 += del * sa * ce + daz * ca;
  v2 -= del * se;
  const float inv = 1.f / sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
  v0 *= inv;
  v1 *= inv;
  v2 *= inv;
  return dt < 1e-4f;
}

// Warp-parallel selection for up to 64 seeds, with the outcome of the
// sequential walk below: every lane finds, for its seeds s, the earlier
// seeds j whose peaks lie within |cos| > 0.99 (a 64-bit mask per seed);
// the kept set is then built in seed order from those masks (a peak is
// kept when it is finite, at or above the threshold and no kept earlier
// peak is in its mask), and the outputs are picked by warp-wide arg-max
// reductions (largest amplitude, or largest |cos| with each target; ties
// go to the earlier seed, as the walk's strict comparisons do).
__device__ __forceinline__ void warp_argmax(float& val, int& idx) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const float v2 = __shfl_xor_sync(0xffffffffu, val, o);
    const int i2 = __shfl_xor_sync(0xffffffffu, idx, o);
    if (v2 > val || (v2 == val && i2 < idx && i2 >= 0) || idx < 0) {
      if (i2 >= 0) {
        val = v2;
        idx = i2;
      }
    }
  }
}

__device__ void select_peaks_warp(const PeakArgs& a, const float* res, long long v, int lane, float* o) {
  uint64_t dup[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int s = lane + 32 * q;
    uint64_t d = 0;
    if (s < a.n_seeds && isfinite(res[4 * s])) {
      const float x = res[4 * s + 1], y = res[4 * s + 2], z = res[4 * s + 3];
      for (int j = 0; j < s; ++j)
        if (isfinite(res[4 * j]) && fabsf(x * res[4 * j + 1] + y * res[4 * j + 2] + z * res[4 * j + 3]) > 0.99f)
          d |= 1ull << j;
    }
    dup[q] = d;
  }
  uint64_t K = 0;
  for (int s = 0; s < a.n_seeds; ++s) {
    const uint64_t mine = (s >> 5) ? dup[1] : dup[0];
    const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)mine, s & 31);
    const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(mine >> 32), s & 31);
    const uint64_t d = ((uint64_t)hi << 32) | lo;
    const float p = res[4 * s];
    if (isfinite(p) && !(d & K) && p >= a.threshold) K |= 1ull << s;
  }
  const int nk = __popcll(K);
  const int nout = nk < a.npeaks ? nk : a.npeaks;
  const bool targets = a.n_targets || a.vtargets;
  uint64_t used = 0;
  int pick[kPkMaxPeaks];
  for (int i = 0; i < nout; ++i) {
    float t0 = 0.f, t1 = 0.f, t2 = 0.f;
    if (targets) {
      if (a.vtargets) {
        const float* t = a.vtargets + v * 3 * a.npeaks + 3 * i;
        const float nrm = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        t0 = t[0] / nrm;
        t1 = t[1] / nrm;
        t2 = t[2] / nrm;
      } else {
        t0 = a.targets[i][0];
        t1 = a.targets[i][1];
        t2 = a.targets[i][2];
      }
    }
    float best = -1.f;
    int bi = -1;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int s = lane + 32 * q;
      if (s < a.n_seeds && ((K >> s) & 1ull) && (targets || !((used >> s) & 1ull))) {
        const float* r = res + 4 * s;
        const float val = targets ? fabsf(t0 * r[1] + t1 * r[2] + t2 * r[3]) : r[0];
        if (targets && !(val > 0.f)) continue;
        if (bi < 0 || val > best) {
          best = val;
          bi = s;
        }
      }
    }
    warp_argmax(best, bi);
    pick[i] = bi;
    if (bi >= 0) used |= 1ull << bi;
  }
  if (lane == 0) {
    for (int i = 0; i < a.npeaks; ++i) {
      if (i < nout && pick[i] >= 0) {
        const float* q = res + 4 * pick[i];
        o[3 * i] = q[0] * q[1];
        o[3 * i + 1] = q[0] * q[2];
        o[3 * i + 2] = q[0] * q[3];
      } else {
        o[3 * i] = o[3 * i + 1] = o[3 * i + 2] = nanf("");
      }
    }
  }
}

template <int L>
__global__ void __launch_bounds__(32 * kPkWarps) sh2peaks_kernel(const __grid_constant__ PeakArgs a) {
  constexpr int NSH = (L + 1) * (L + 2) / 2;
  extern __shared__ __align__(16) float psm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* sh = psm + warp * (NSH + 4 * kPkMaxSeeds);
  float* res = sh + NSH;  // [n_seeds][4]: amplitude, direction
  const float fnan = nanf("");
  for (long long v = (long long)blockIdx.x * kPkWarps + warp; v < a.n; v += (long long)gridDim.x * kPkWarps) {
    float* o = a.out + v * 3 * a.npeaks;
    // check_input (sh2peaks.cpp:277-299) + the masked voxels' NaN input (:134-138)
    bool skip = a.mask && !a.mask[v];
    bool iso = true;
    for (int c = lane; c < NSH; c += 32) {
      const float x = a.sh[v * a.stride + c];
      sh[c] = x;
      if (isnan(x)) skip = true;
      if (c && x != 0.f) iso = false;
    }
    if (a.vtargets && isnan(a.vtargets[v * 3 * a.npeaks])) skip = true;
    skip = __any_sync(0xffffffffu, skip) || __all_sync(0xffffffffu, iso);
    if (skip) {
      for (int i = lane; i < 3 * a.npeaks; i += 32) o[i] = fnan;
      continue;
    }
    __syncwarp();
    {
      // the searches, one Newton step per lane per round: a lane whose seed's
      // search ends (converged, or 50 steps without converging: NaN) stores
      // it and takes the next unassigned seed, so the warp's lanes stay busy
      // until the seeds run out instead of waiting, seed by seed, for the
      // longest search of each group of 32
      int s = lane, steps = 0, next = 32;
      float v0 = 0.f, v1 = 0.f, v2 = 1.f;
      if (s < a.n_seeds) {
        v0 = a.seeds[s][0];
        v1 = a.seeds[s][1];
        v2 = a.seeds[s][2];
      }
      while (__any_sync(0xffffffffu, s < a.n_seeds)) {
        bool fin = false;
        if (s < a.n_seeds) {
          float amp;
          const bool done = peak_step<L>(sh, v0, v1, v2, a.plm_k, amp);
          if (done || ++steps == 50) {
            if (!done) amp = v0 = v1 = v2 = fnan;
            res[4 * s] = amp;
            res[4 * s + 1] = v0;
            res[4 * s + 2] = v1;
            res[4 * s + 3] = v2;
            fin = true;
          }
        }
        const unsigned f = __ballot_sync(0xffffffffu, fin);
        if (fin) {
          s = next + __popc(f & ((1u << lane) - 1u));
          steps = 0;
          if (s < a.n_seeds) {
            v0 = a.seeds[s][0];
            v1 = a.seeds[s][1];
            v2 = a.seeds[s][2];
          }
        }
        next += __popc(f);
      }
    }
    __syncwarp();
    if (a.n_seeds <= 64) {
      select_peaks_warp(a, res, v, lane, o);
    } else if (lane == 0) {
      // peaks in seed order, duplicates (|cos| > 0.99 with a kept one) and
      // those below the threshold dropped; kept indices go back into res
      int kept[kPkMaxSeeds];
      int nk = 0;
      for (int s = 0; s < a.n_seeds; ++s) {
        const float p = res[4 * s];
        if (!isfinite(p)) continue;
        bool dup = false;
        for (int j = 0; j < nk && !dup; ++j) {
          const float* q = res + 4 * kept[j];
          dup = fabsf(res[4 * s + 1] * q[1] + res[4 * s + 2] * q[2] + res[4 * s + 3] * q[3]) > 0.99f;
        }
        if (!dup && p >= a.threshold) kept[nk++] = s;
      }
      const int nout = nk < a.npeaks ? nk : a.npeaks;
      int pick[kPkMaxPeaks];
      if (a.n_targets || a.vtargets) {
        for (int i = 0; i < nout; ++i) {
          float t0, t1, t2;
          if (a.vtargets) {
            const float* t = a.vtargets + v * 3 * a.npeaks + 3 * i;
            const float nrm = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
            t0 = t[0] / nrm;
            t1 = t[1] / nrm;
            t2 = t[2] / nrm;
          } else {
            t0 = a.targets[i][0];
            t1 = a.targets[i][1];
            t2 = a.targets[i][2];
          }
          float mdot = 0.f;
          pick[i] = -1;
          for (int j = 0; j < nk; ++j) {
            const float* q = res + 4 * kept[j];
            const float f = fabsf(t0 * q[1] + t1 * q[2] + t2 * q[3]);
            if (f > mdot) {
              mdot = f;
              pick[i] = kept[j];
            }
          }
        }
      } else {
        // largest amplitudes first (partial_sort_copy with a > b); equal
        // amplitudes keep seed order
        for (int i = 0; i < nout; ++i) {
          int best = -1;
          for (int j = 0; j < nk; ++j) {
            bool used = false;
            for (int u = 0; u < i; ++u) used = used || pick[u] == kept[j];
            if (!used && (best < 0 || res[4 * kept[j]] > res[4 * best])) best = kept[j];
          }
          pick[i] = best;
        }
      }
      for (int i = 0; i < a.npeaks; ++i) {
        if (i < nout && pick[i] >= 0) {
          const float* q = res + 4 * pick[i];
          o[3 * i] = q[0] * q[1];
          o[3 * i + 1] = q[0] * q[2];
          o[3 * i + 2] = q[0] * q[3];
        } else {
          o[3 * i] = o[3 * i + 1] = o[3 * i + 2] = fnan;
        }
      }
    }
    __syncwarp();
  }
}

template <int L>
int launch(const PeakArgs& a, cudaStream_t s) {
  constexpr int NSH = (L + 1) * (L + 2) / 2;
  const size_t smem = (size_t)kPkWarps * (NSH + 4 * kPkMaxSeeds) * sizeof(float);
  int dev = 0, nsm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(sh2peaks_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_sh2peaks: ") + cudaGetErrorString(e));
  const long long blocks = std::min<long long>((a.n + kPkWarps - 1) / kPkWarps, (long long)nsm * 16);
  sh2peaks_kernel<L><<<(unsigned)std::max<long long>(blocks, 1), 32 * kPkWarps, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_sh2peaks: ") + cudaGetErrorString(e));
  return CSD_OK;
}

}  // namespace

extern "C" int csd_sh2peaks(const float* sh, int64_t n_voxels, int64_t voxel_stride, int lmax, const uint8_t* mask,
                            const float* seeds_azel, int n_seeds, int npeaks, float threshold,
                            const float* directions, int n_directions, const float* peaks_in, float* peaks_out,
                            void* stream) {
  if (n_voxels < 0 || (n_voxels > 0 && (!sh || !peaks_out)) || npeaks < 1 || npeaks > kPkMaxPeaks ||
      n_seeds < 1 || n_seeds > kPkMaxSeeds || !seeds_azel || n_directions < 0 || n_directions > kPkMaxPeaks ||
      (n_directions && (!directions || n_directions != npeaks)) || (peaks_in && n_directions) ||
      voxel_stride < (lmax + 1) * (lmax + 2) / 2)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_sh2peaks: invalid argument");
  if (n_voxels == 0) return CSD_OK;
  PeakArgs a{};
  a.sh = sh;
  a.n = n_voxels;
  a.stride = voxel_stride;
  a.mask = mask;
  a.vtargets = peaks_in;
  a.out = peaks_out;
  a.n_seeds = n_seeds;
  a.npeaks = npeaks;
  a.n_targets = n_directions;
  a.threshold = threshold;
  plm_start_table(a.plm_k, 12);
  for (int i = 0; i < n_seeds; ++i) {
    // Direction(phi, theta) (sh2peaks.cpp:104), in float as the reference
    const float phi = seeds_azel[2 * i], theta = seeds_azel[2 * i + 1];
    a.seeds[i][0] = std::cos(phi) * std::sin(theta);
    a.seeds[i][1] = std::sin(phi) * std::sin(theta);
    a.seeds[i][2] = std::cos(theta);
  }
  for (int i = 0; i < n_directions; ++i) {
    const float* d = directions + 3 * i;
    const float nrm = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) a.targets[i][k] = d[k] / nrm;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  switch (lmax) {
    case 2: return launch<2>(a, s);
    case 4: return launch<4>(a, s);
    case 6: return launch<6>(a, s);
    case 8: return launch<8>(a, s);
    case 10: return launch<10>(a, s);
    case 12: return launch<12>(a, s);
    default: return csdb200::set_error(CSD_ERR_UNSUPPORTED, "csd_sh2peaks: lmax must be even, 2..12");
  }
}
