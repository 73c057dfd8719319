// fod2fixel's FMLS segmenter on the GPU (MRtrix3 src/dwi/fmls.cpp:118-311).
//
// One warp a voxel.  The lanes compute the voxel's amplitudes on the ndir
// (1281) directions in FP64 (SH -> amplitude matrix, L2-resident) into
// shared memory and sort the direction indices by |amplitude| descending,
// index ascending (the reference's multimap order), by a bitonic network
// over the next power of two in shared memory.  Lane 0 then grows the lobes
// (fmls_core.cuh: the region growing and the pending assignments) with the
// direction labels and the lobes' state in the warp's shared memory (up to
// kFmlsLobes lobes; a voxel that makes more is grown again from its global
// slot).  The Newton refinements of the candidate peaks are independent of
// one another, so the lanes compute them in parallel, and lane 0 finishes
// the lobes (thresholds, the nearest-peak test, the fixels) from those
// results.  The core is the same source the CPU tests build for the host and
// compare with the oracle.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/csd_b200.h"
#include "fmls_core.cuh"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu
}

namespace {

constexpr int kFmlsWarps = 1;  // ~38 KB of shared memory a warp: five warps an SM
constexpr int kFmlsMaxSort = 2048;  // directions at most (the sort's width)
constexpr int kFmlsMaxNsh = 153;    // lmax 16
constexpr int kFmlsLobes = 128;     // lobes a voxel may create in shared memory (more: the global slot)

int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

// per warp slot in global memory: ints label parent neg head tail next
// retro_dir retro_lobe, doubles max_peak mean(3) integral peak_dir(3) -- one
// entry per direction; the shared-memory lobes use only the retro lists
constexpr int kSlotInts = 8, kSlotDoubles = 8;

// Shared memory of one warp: values [nd] and sh [nsh] doubles, the sort keys
// [sort_n] and labels [nd] ints, then for kFmlsLobes lobes the ints parent
// neg head tail next and the doubles max_peak integral mean(3) peak_dir(3)
// and the refined peaks' values (1) and directions (3).
__host__ __device__ inline size_t fmls_warp_bytes(int nd, int nsh, int sort_n) {
  const size_t a = ((size_t)(nd + nsh) * sizeof(double) + (size_t)(sort_n + nd) * sizeof(int) + 15) & ~(size_t)15;
  return a + (size_t)5 * kFmlsLobes * sizeof(int) + (size_t)12 * kFmlsLobes * sizeof(double);
}

struct FmlsArgs {
  fmls::Tables t;
  const float* fod;
  long long n, vs, cs;
  const uint8_t* mask;
  int max_fixels;
  int32_t* counts;
  float* fixels;
  char* scratch;
  long long slot_bytes;
  int sort_n;
};

__global__ void __launch_bounds__(kFmlsWarps * 32) fmls_segment_kernel(const __grid_constant__ FmlsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nd = a.t.ndir, nsh = a.t.nsh;
  unsigned char* base = smem_raw + wib * fmls_warp_bytes(nd, nsh, a.sort_n);
  double* values = reinterpret_cast<double*>(base);
  double* sh = values + nd;
  int* keys = reinterpret_cast<int*>(sh + nsh);
  int* slabel = keys + a.sort_n;
  int* li = reinterpret_cast<int*>(base + (((size_t)(nd + nsh) * sizeof(double) +
                                            (size_t)(a.sort_n + nd) * sizeof(int) + 15) & ~(size_t)15));
  double* ld = reinterpret_cast<double*>(li + 5 * kFmlsLobes);
  double* pre_val = ld + 8 * kFmlsLobes;
  double* pre_u = pre_val + kFmlsLobes;

  const long long gw = (long long)blockIdx.x * kFmlsWarps + wib;
  char* slot = a.scratch + gw * a.slot_bytes;
  int* ib = reinterpret_cast<int*>(slot);
  double* db = reinterpret_cast<double*>(slot + (((size_t)kSlotInts * nd * sizeof(int) + 15) & ~(size_t)15));
  // the global slot's workspace (every array one entry per direction)
  fmls::Work wg;
  wg.values = values;
  wg.order = keys;
  wg.label = ib;
  wg.parent = ib + nd;
  wg.neg = ib + 2 * nd;
  wg.peak_head = ib + 3 * nd;
  wg.peak_tail = ib + 4 * nd;
  wg.peak_next = ib + 5 * nd;
  wg.retro_dir = ib + 6 * nd;
  wg.retro_lobe = ib + 7 * nd;
  wg.max_peak = db;
  wg.mean = db + nd;
  wg.integral = db + 4 * nd;
  wg.peak_dir = db + 5 * nd;
  // the shared-memory workspace: labels and up to kFmlsLobes lobes
  fmls::Work ws = wg;
  ws.label = slabel;
  ws.parent = li;
  ws.neg = li + kFmlsLobes;
  ws.peak_head = li + 2 * kFmlsLobes;
  ws.peak_tail = li + 3 * kFmlsLobes;
  ws.peak_next = li + 4 * kFmlsLobes;
  ws.max_peak = ld;
  ws.integral = ld + kFmlsLobes;
  ws.mean = ld + 2 * kFmlsLobes;
  ws.peak_dir = ld + 5 * kFmlsLobes;

  const long long nwarps = (long long)gridDim.x * kFmlsWarps;
  for (long long v = gw; v < a.n; v += nwarps) {
    if (a.mask && !a.mask[v]) {
      if (lane == 0) a.counts[v] = 0;
      continue;
    }
    const float* src = a.fod + v * a.vs;
    for (int k = lane; k < nsh; k += 32) sh[k] = (double)src[(long long)k * a.cs];
    __syncwarp();
    if (fmls::skip_voxel(sh, nsh)) {
      __syncwarp();
      if (lane == 0) a.counts[v] = 0;
      continue;
    }
    for (int d = lane; d < nd; d += 32) {
      const double* row = a.t.sh2amp + (long long)d * nsh;
      double s = 0.0;
      for (int k = 0; k < nsh; ++k) s = fma(__ldg(row + k), sh[k], s);
      values[d] = s;
    }
    for (int i = lane; i < a.sort_n; i += 32) keys[i] = i;
    __syncwarp();
    // bitonic sort of keys in the segmenter's order (padding keys >= nd last)
    for (int k = 2; k <= a.sort_n; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = lane; i < a.sort_n; i += 32) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const int ka = keys[i], kb = keys[ixj];
            const bool up = (i & k) == 0;
            if (up ? fmls::before(values, nd, kb, ka) : fmls::before(values, nd, ka, kb)) {
              keys[i] = kb;
              keys[ixj] = ka;
            }
          }
        }
        __syncwarp();
      }
    }
    // lane 0: the region growing and the pending assignments
    int nl = 0;
    bool in_smem = true;
    if (lane == 0 && values[keys[0]] > 0.0) {
      int nr = 0;
      nl = fmls::grow(a.t, ws, &nr, kFmlsLobes);
      if (nl < 0) {  // more lobes than the shared arrays hold
        in_smem = false;
        nl = fmls::grow(a.t, wg, &nr);
      }
      fmls::assign_pending(a.t, in_smem ? ws : wg, nr);
    }
    nl = __shfl_sync(0xffffffffu, nl, 0);
    in_smem = __shfl_sync(0xffffffffu, in_smem ? 1 : 0, 0) != 0;
    if (nl == 0) {
      if (lane == 0) a.counts[v] = 0;
      __syncwarp();
      continue;
    }
    __syncwarp();
    const fmls::Work& w = in_smem ? ws : wg;
    // the candidate peaks' Newton refinements, spread over the lanes (in the
    // global slot's case lane 0 refines them itself, in finish_lobes)
    if (in_smem) {
      for (int p = lane; p < nl; p += 32) {
        if (!fmls::peak_candidate(a.t, w, p)) continue;
        double u[3] = {w.peak_dir[3 * p], w.peak_dir[3 * p + 1], w.peak_dir[3 * p + 2]};
        pre_val[p] = fmls::get_peak(a.t, sh, u);
        for (int k = 0; k < 3; ++k) pre_u[3 * p + k] = u[k];
      }
    }
    __syncwarp();
    if (lane == 0)
      a.counts[v] = fmls::finish_lobes(a.t, w, sh, nl,
                                       reinterpret_cast<fmls::Fixel*>(a.fixels + v * (long long)a.max_fixels * 8),
                                       a.max_fixels, in_smem ? pre_val : nullptr, in_smem ? pre_u : nullptr);
    __syncwarp();
  }
}

template <class T>
cudaError_t upload(T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMalloc(dst, n * sizeof(T));
  if (e == cudaSuccess) e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

}  // namespace

struct csd_fmls {
  int device = 0;
  fmls::Tables t{};  // device pointers
  double *unit = nullptr, *weight = nullptr, *sh2amp = nullptr, *al = nullptr;
  int32_t *adj_off = nullptr, *adj = nullptr, *grid_off = nullptr, *grid = nullptr;
  char* scratch = nullptr;
  size_t scratch_warps = 0;
};

extern "C" void csd_fmls_destroy(csd_fmls* p) {
  if (!p) return;
  cudaFree(p->unit);
  cudaFree(p->weight);
  cudaFree(p->sh2amp);
  cudaFree(p->al);
  cudaFree(p->adj_off);
  cudaFree(p->adj);
  cudaFree(p->grid_off);
  cudaFree(p->grid);
  cudaFree(p->scratch);
  delete p;
}

extern "C" int csd_fmls_create(const csd_fmls_tables* c, csd_fmls** out) {
  if (!c || !out) return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: null argument");
  *out = nullptr;
  const int nd = c->ndir;
  const long long ncell = (long long)c->num_az * c->num_el;
  if (nd < 2 || nd > kFmlsMaxSort || c->lmax < 0 || c->lmax > 16 || (c->lmax & 1) ||
      c->nsh != (c->lmax + 1) * (c->lmax + 2) / 2 || c->nsh > kFmlsMaxNsh || !c->unit || !c->weight ||
      !c->adj_off || !c->adj || !c->sh2amp || !c->al || c->al_ndir < 2 || c->n_al != (c->lmax / 2 + 1) * (c->lmax / 2 + 1) ||
      !(c->al_inc > 0.0) || c->num_az < 2 || c->num_el < 2 || !(c->az_step > 0.0) || !(c->el_step > 0.0) ||
      !c->grid_off || !c->grid || !(c->merge_ratio >= 0.0))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: invalid tables");
  // the kernel reads these without further checks
  if (c->adj_off[0] != 0 || c->adj_off[nd] != c->n_adj || c->grid_off[0] != 0 || c->grid_off[ncell] != c->n_grid)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: inconsistent offsets");
  for (int d = 0; d < nd; ++d) {
    const int deg = c->adj_off[d + 1] - c->adj_off[d];
    if (deg < 0 || deg > fmls::kMaxAdj)
      return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: a direction has more than 16 neighbours");
  }
  for (int e = 0; e < c->n_adj; ++e)
    if (c->adj[e] < 0 || c->adj[e] >= nd) return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: bad neighbour");
  for (long long q = 0; q < ncell; ++q)
    if (c->grid_off[q + 1] <= c->grid_off[q])
      return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: an empty grid cell");
  for (int e = 0; e < c->n_grid; ++e)
    if (c->grid[e] < 0 || c->grid[e] >= nd) return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create: bad grid entry");
  csd_fmls* p = new csd_fmls();
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = upload(&p->unit, c->unit, 3 * (size_t)nd);
  if (e == cudaSuccess) e = upload(&p->weight, c->weight, (size_t)nd);
  if (e == cudaSuccess) e = upload(&p->sh2amp, c->sh2amp, (size_t)nd * c->nsh);
  if (e == cudaSuccess) e = upload(&p->al, c->al, (size_t)c->al_ndir * c->n_al);
  if (e == cudaSuccess) e = upload(&p->adj_off, c->adj_off, (size_t)nd + 1);
  if (e == cudaSuccess) e = upload(&p->adj, c->adj, (size_t)c->n_adj);
  if (e == cudaSuccess) e = upload(&p->grid_off, c->grid_off, (size_t)ncell + 1);
  if (e == cudaSuccess) e = upload(&p->grid, c->grid, (size_t)c->n_grid);
  if (e != cudaSuccess) {
    csd_fmls_destroy(p);
    return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_create: ") + cudaGetErrorString(e));
  }
  p->t = fmls::Tables{nd, c->lmax, c->nsh, p->unit, p->weight, p->adj_off, p->adj, p->sh2amp, c->al_ndir, c->n_al,
                      c->al_inc, p->al, c->num_az, c->num_el, c->az_begin, c->el_begin, c->az_step, c->el_step,
                      p->grid_off, p->grid, c->integral_threshold, c->peak_value_threshold, c->merge_ratio};
  *out = p;
  return CSD_OK;
}

extern "C" int csd_fmls_segment(csd_fmls* p, const float* fod, int64_t n, int64_t voxel_stride, int64_t coef_stride,
                                const uint8_t* mask, int max_fixels, int32_t* counts, float* fixels, void* stream) {
  if (!p || n < 0 || max_fixels < 1 || (n > 0 && (!fod || !counts || !fixels)))
    return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_segment: invalid argument");
  if (n == 0) return CSD_OK;
  const int nd = p->t.ndir, nsh = p->t.nsh, sort_n = next_pow2(nd);
  const size_t smem = kFmlsWarps * fmls_warp_bytes(nd, nsh, sort_n);
  int nsm = 0, smem_max = 0, per_sm = 0;
  cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, p->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device);
  if (e == cudaSuccess && smem > (size_t)smem_max)
    return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_segment: direction set too large for shared memory");
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fmls_segment_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fmls_segment_kernel, kFmlsWarps * 32, smem);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
  const long long blocks = std::max<long long>(
      1, std::min<long long>((n + kFmlsWarps - 1) / kFmlsWarps, (long long)nsm * std::max(1, per_sm)));
  const size_t slot_bytes = ((((size_t)kSlotInts * nd * sizeof(int) + 15) & ~(size_t)15) +
                             (size_t)kSlotDoubles * nd * sizeof(double) + 255) & ~(size_t)255;
  const size_t warps = (size_t)blocks * kFmlsWarps;
  if (warps > p->scratch_warps) {
    cudaFree(p->scratch);
    p->scratch = nullptr;
    p->scratch_warps = 0;
    e = cudaMalloc(&p->scratch, warps * slot_bytes);
    if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
    p->scratch_warps = warps;
  }
  FmlsArgs a{p->t, fod, n, voxel_stride, coef_stride, mask, max_fixels, counts, fixels, p->scratch,
             (long long)slot_bytes, sort_n};
  fmls_segment_kernel<<<(unsigned)blocks, kFmlsWarps * 32, smem, static_cast<cudaStream_t>(stream)>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
  return CSD_OK;
}
