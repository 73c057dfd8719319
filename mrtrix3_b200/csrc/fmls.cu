// fod2fixel's FMLS segmenter on the GPU (MRtrix3 src/dwi/fmls.cpp:118-311).
//
// The voxels go in rounds of kFmlsChunk, each round three kernels:
// - fmls_segment_kernel, a warp a voxel: the amplitudes on the ndir (1281)
//   directions in FP64 (the SH -> amplitude matrix transposed, L2-resident)
//   into the warp's global slot, their 64-bit sort keys sorted by a bitonic
//   network in shared memory into the reference's multimap order
//   (|amplitude| descending, index ascending), the lobes grown by the warp
//   (grow_warp: the lanes look up a direction's neighbours, warp reductions
//   decide, lane 0 applies the core's step) with 8-bit labels and up to
//   kFmlsLobes lobes in shared memory, and lane 0's pending assignments.
//   It leaves the voxel's state (labels, lobes) in global memory and lists
//   the candidate peaks.  A voxel that makes more lobes is grown again and
//   finished by lane 0 on its global slot.
// - fmls_peak_kernel, a thread a listed peak: the Newton refinements, which
//   are independent of one another (a peak's start changes only when that
//   peak itself is refined).  A thread takes the next peak as soon as its
//   own is done, so no voxel waits for its slowest peak.
// - fmls_finish_kernel, a thread a voxel: thresholds, the nearest-peak test
//   and the fixels from the refined peaks.
// The core is the same source the CPU tests build for the host and compare
// with the oracle.
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

// Optional per-phase cycle counters of fmls_segment_kernel (build with
// -DCSD_PHASE_TIMERS): lane 0 of each warp adds clock64() deltas of
// amplitudes / sort / growing / pending assignments / state out to
// g_fmls_cycles.
#ifdef CSD_PHASE_TIMERS
__device__ unsigned long long g_fmls_cycles[8];
#define FMLS_T(var) const long long var = clock64()
#define FMLS_ACC(idx, a, b) if (lane == 0) atomicAdd(&g_fmls_cycles[idx], (unsigned long long)((b) - (a)))
#else
#define FMLS_T(var)
#define FMLS_ACC(idx, a, b)
#endif

namespace {

constexpr int kFmlsWarps = 1;       // one warp a block (occupancy is set by shared memory)
constexpr int kFmlsMaxSort = 2048;  // directions at most (the sort's width; the keys carry 11 index bits)
constexpr int kFmlsMaxNsh = 153;    // lmax 16
constexpr int kFmlsLobes = 120;     // lobes a voxel may create in shared memory (8-bit links; more: the global slot)

// the shared-memory workspace (8-bit labels and lobe links, 16-bit order)
// and the global slot's (32-bit), which shares the order in shared memory
using WorkS = fmls::WorkT<int8_t, uint16_t>;
using WorkG = fmls::WorkT<int, uint16_t>;

int next_pow2(int n) {
  int p = 1;
  while (p < n) p <<= 1;
  return p;
}

__host__ __device__ constexpr size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// per warp slot in global memory: ints label parent neg head tail next
// retro_dir retro_lobe, doubles values max_peak mean(3) integral peak_dir(3)
// -- one entry per direction; the shared-memory path uses the values and the
// retro lists only
constexpr int kSlotInts = 8, kSlotDoubles = 9;

// Shared memory of one warp: sh [nsh] doubles, then one region that holds
// the sort keys [sort_n] (64-bit) while sorting and afterwards the order
// [nd] (16-bit), the labels [nd] (8-bit), the lobes' links parent neg head
// tail next [kFmlsLobes] (8-bit) and their doubles max_peak integral mean(3)
// peak_dir(3) and the refined peaks' values (1) and directions (3).
__host__ __device__ inline size_t fmls_after_sort_bytes(int nd) {
  return align16((size_t)nd * 2) + align16((size_t)nd) + align16((size_t)5 * kFmlsLobes) +
         (size_t)12 * kFmlsLobes * sizeof(double);
}
__host__ __device__ inline size_t fmls_region_bytes(int nd, int sort_n) {
  const size_t k = (size_t)sort_n * 8, b = fmls_after_sort_bytes(nd);
  return align16(k > b ? k : b);
}
__host__ __device__ inline size_t fmls_warp_bytes(int nd, int nsh, int sort_n) {
  return align16((size_t)nsh * sizeof(double)) + fmls_region_bytes(nd, sort_n);
}

// A voxel's state between the kernels, laid out as the tail of the growing
// kernel's shared region (from the labels on): 8-bit labels [nd], the
// lobes' 8-bit links (5 x kFmlsLobes), their doubles max_peak integral
// mean(3) peak_dir(3), and the refined peaks' values (1) and directions (3).
__host__ __device__ inline size_t fmls_state_bytes(int nd) {
  return align16((size_t)nd) + align16((size_t)5 * kFmlsLobes) + (size_t)12 * kFmlsLobes * sizeof(double);
}
struct StateView {
  WorkS w;
  double* pre_val;
  double* pre_u;
};
__device__ inline StateView state_view(unsigned char* st, int nd) {
  StateView s{};
  s.w.label = reinterpret_cast<int8_t*>(st);
  int8_t* links = s.w.label + align16((size_t)nd);
  s.w.parent = links;
  s.w.neg = links + kFmlsLobes;
  s.w.peak_head = links + 2 * kFmlsLobes;
  s.w.peak_tail = links + 3 * kFmlsLobes;
  s.w.peak_next = links + 4 * kFmlsLobes;
  double* ld = reinterpret_cast<double*>(links + align16((size_t)5 * kFmlsLobes));
  s.w.max_peak = ld;
  s.w.integral = ld + kFmlsLobes;
  s.w.mean = ld + 2 * kFmlsLobes;
  s.w.peak_dir = ld + 5 * kFmlsLobes;
  s.pre_val = ld + 8 * kFmlsLobes;
  s.pre_u = ld + 9 * kFmlsLobes;
  return s;
}

constexpr int kFmlsChunk = 16384;   // voxels per round of the three kernels
constexpr int kPeakThreads = 128;   // threads a block of the peak kernel
constexpr int kPeakShift = 7;       // a listed peak is (voxel in the round) << 7 | peak

// fmls::grow (fmls.cpp:178-246) with the warp: for each direction in order,
// lane e looks up the lobe of neighbour e (its label's root, if that lobe's
// sign matches); two warp reductions give the smallest and largest adjacent
// lobe, which decide the common steps (no adjacent lobe: a new one; one: an
// addition), and lane 0 applies the step with the arithmetic of the core's
// lobe constructor and lobe_add.  With two or more adjacent lobes the merge
// test reads the largest (the last in ascending order), and the merges into
// the smallest run in ascending order, each next lobe found by another
// reduction -- the order of fmls::grow, so every value is computed as there.
// The order is fixed once sorted, so the global tables a step reads (the
// direction's value, neighbour list, unit vector and weight) are fetched one
// and two steps ahead: only the labels and lobes (shared memory) depend on
// earlier steps.  Returns the lobes created, -1 past max_lobes.
template <class W>
__device__ int grow_warp(const fmls::Tables& t, const W& w, int* n_retro, int max_lobes, int lane) {
  const int nd = t.ndir;
  for (int d = lane; d < nd; d += 32) w.label[d] = -1;
  __syncwarp();
  // step k's inputs (c), step k + 1's neighbour offsets (n), step k + 2's (nn)
  int dc = w.order[0];
  int e0 = __ldg(t.adj_off + dc), degc = __ldg(t.adj_off + dc + 1) - e0;
  int nbc = lane < degc ? __ldg(t.adj + e0 + lane) : 0;
  double uc0 = __ldg(t.unit + 3 * dc), uc1 = __ldg(t.unit + 3 * dc + 1), uc2 = __ldg(t.unit + 3 * dc + 2);
  double wc = __ldg(t.weight + dc);
  double vc = w.values[dc];
  int dn = nd > 1 ? w.order[1] : 0;
  int e0n = __ldg(t.adj_off + dn), degn = __ldg(t.adj_off + dn + 1) - e0n;
  int nl = 0, nr = 0;
  for (int k = 0; k < nd; ++k) {
    // fetch ahead: step k + 1's neighbours, value, direction and weight; step k + 2's offsets
    const int nbn = (k + 1 < nd && lane < degn) ? __ldg(t.adj + e0n + lane) : 0;
    const double un0 = __ldg(t.unit + 3 * dn), un1 = __ldg(t.unit + 3 * dn + 1), un2 = __ldg(t.unit + 3 * dn + 2);
    const double wn = __ldg(t.weight + dn);
    const double vn = w.values[dn];
    const int dnn = k + 2 < nd ? w.order[k + 2] : 0;
    const int e0nn = __ldg(t.adj_off + dnn), degnn = __ldg(t.adj_off + dnn + 1) - e0nn;
    // step k
    const int d = dc;
    const double v = vc;
    const int vneg = v <= 0.0 ? 1 : 0;
    int r = -1;
    if (lane < degc) {
      const int lab = w.label[nbc];
      if (lab >= 0) {
        r = fmls::root(w, lab);
        if (w.neg[r] != vneg) r = -1;
      }
    }
    const int rmax = __reduce_max_sync(0xffffffffu, r);
    bool add = false;
    int a0 = -1;
    if (rmax < 0) {
      if (nl >= max_lobes) return -1;
      if (lane == 0) {
        // FOD_lobe constructor (fmls.h:60-72)
        const double av = fabs(v);
        w.parent[nl] = nl;
        w.neg[nl] = vneg;
        w.max_peak[nl] = av;
        w.peak_head[nl] = w.peak_tail[nl] = nl;
        w.peak_next[nl] = -1;
        w.peak_dir[3 * nl] = uc0;
        w.peak_dir[3 * nl + 1] = uc1;
        w.peak_dir[3 * nl + 2] = uc2;
        w.mean[3 * nl] = uc0 * av * wc;
        w.mean[3 * nl + 1] = uc1 * av * wc;
        w.mean[3 * nl + 2] = uc2 * av * wc;
        w.integral[nl] = fabs(v * wc);
        w.label[d] = nl;
      }
      ++nl;
    } else {
      // the smallest adjacent lobe (no lobe reads as 0xffffffff)
      a0 = (int)__reduce_min_sync(0xffffffffu, (unsigned)r);
      if (a0 == rmax) {
        add = true;
      } else if (fabs(v) / w.max_peak[rmax] > t.merge_ratio) {
        for (int cur = a0;;) {
          const unsigned nx = __reduce_min_sync(0xffffffffu, r > cur ? (unsigned)r : 0xffffffffu);
          if (nx == 0xffffffffu) break;
          if (lane == 0) fmls::lobe_merge(w, a0, (int)nx);
          __syncwarp();
          cur = (int)nx;
        }
        add = true;
      } else {
        if (lane == 0) {
          w.retro_dir[nr] = d;
          w.retro_lobe[nr] = a0;
        }
        ++nr;
      }
    }
    if (add && lane == 0) {
      // FOD_lobe::add (fmls.h:82-91), as fmls::lobe_add
      double* m = w.mean + 3 * a0;
      w.label[d] = a0;
      const double mult = (m[0] * uc0 + m[1] * uc1 + m[2] * uc2) > 0.0 ? 1.0 : -1.0;
      const double av = fabs(v);
      m[0] += uc0 * mult * av * wc;
      m[1] += uc1 * mult * av * wc;
      m[2] += uc2 * mult * av * wc;
      w.integral[a0] += fabs(v * wc);
    }
    __syncwarp();
    dc = dn;
    degc = degn;
    nbc = nbn;
    uc0 = un0;
    uc1 = un1;
    uc2 = un2;
    wc = wn;
    vc = vn;
    dn = dnn;
    e0n = e0nn;
    degn = degnn;
  }
  *n_retro = nr;
  return nl;
}

// The sort key of direction d with amplitude v: |v|'s bits above the lowest
// 11 (an order-preserving integer for a non-negative double), then 2047 - d,
// so that a larger key comes first in the segmenter's order (|value|
// descending, index ascending) whenever the truncated magnitudes differ or
// are equal exactly.
__device__ __forceinline__ unsigned long long sort_key(double v, int d) {
  return ((unsigned long long)__double_as_longlong(fabs(v)) & ~0x7FFull) | (unsigned long long)(0x7FF - d);
}
__device__ __forceinline__ int key_dir(unsigned long long k) { return 0x7FF - (int)(k & 0x7FF); }

struct FmlsArgs {
  fmls::Tables t;
  const float* fod;
  long long n, vs, cs;  // voxels, voxel stride, coefficient stride
  const uint8_t* mask;
  int max_fixels;
  int32_t* counts;
  float* fixels;
  char* scratch;        // per-warp slots of the growing kernel
  long long slot_bytes;
  int sort_n;
  long long v0;         // this round's first voxel; n - v0 > nc ... the round is [v0, v0 + nc)
  int nc;
  unsigned char* state;  // [nc] voxel states (fmls_state_bytes each)
  int* vnl;              // [nc] lobes left to finish (0: written already)
  int* peaks;            // [nc * kFmlsLobes] listed candidate peaks
  int* counters;         // [0] peaks listed, [1] peaks taken by the peak kernel
};

__global__ void __launch_bounds__(kFmlsWarps * 32, 12) fmls_segment_kernel(const __grid_constant__ FmlsArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nd = a.t.ndir, nsh = a.t.nsh, sort_n = a.sort_n;
  unsigned char* base = smem_raw + wib * fmls_warp_bytes(nd, nsh, sort_n);
  double* sh = reinterpret_cast<double*>(base);
  unsigned char* region = base + align16((size_t)nsh * sizeof(double));
  unsigned long long* keys = reinterpret_cast<unsigned long long*>(region);
  uint16_t* order = reinterpret_cast<uint16_t*>(region);
  int8_t* slabel = reinterpret_cast<int8_t*>(region + align16((size_t)nd * 2));
  int8_t* links = slabel + align16((size_t)nd);
  double* ld = reinterpret_cast<double*>(links + align16((size_t)5 * kFmlsLobes));

  const long long gw = (long long)blockIdx.x * kFmlsWarps + wib;
  char* slot = a.scratch + gw * a.slot_bytes;
  int* ib = reinterpret_cast<int*>(slot);
  double* db = reinterpret_cast<double*>(slot + align16((size_t)kSlotInts * nd * sizeof(int)));
  double* values = db;  // the amplitudes, in the slot (read in order by the growing)
  // the global slot's workspace (every array one entry per direction)
  WorkG wg;
  wg.values = values;
  wg.order = order;
  wg.label = ib;
  wg.parent = ib + nd;
  wg.neg = ib + 2 * nd;
  wg.peak_head = ib + 3 * nd;
  wg.peak_tail = ib + 4 * nd;
  wg.peak_next = ib + 5 * nd;
  wg.retro_dir = ib + 6 * nd;
  wg.retro_lobe = ib + 7 * nd;
  wg.max_peak = db + nd;
  wg.mean = db + 2 * nd;
  wg.integral = db + 5 * nd;
  wg.peak_dir = db + 6 * nd;
  // the shared-memory workspace: labels and up to kFmlsLobes lobes
  WorkS ws;
  ws.values = values;
  ws.order = order;
  ws.label = slabel;
  ws.parent = links;
  ws.neg = links + kFmlsLobes;
  ws.peak_head = links + 2 * kFmlsLobes;
  ws.peak_tail = links + 3 * kFmlsLobes;
  ws.peak_next = links + 4 * kFmlsLobes;
  ws.retro_dir = wg.retro_dir;
  ws.retro_lobe = wg.retro_lobe;
  ws.max_peak = ld;
  ws.integral = ld + kFmlsLobes;
  ws.mean = ld + 2 * kFmlsLobes;
  ws.peak_dir = ld + 5 * kFmlsLobes;

  const size_t sb = fmls_state_bytes(nd);
  const long long nwarps = (long long)gridDim.x * kFmlsWarps;
  for (long long c = gw; c < a.nc; c += nwarps) {
    const long long v = a.v0 + c;
    if (lane == 0) a.vnl[c] = 0;
    if (a.mask && !a.mask[v]) {
      if (lane == 0) a.counts[v] = 0;
      continue;
    }
    const float* src = a.fod + v * a.vs;
    __syncwarp();  // the previous voxel's last reads of the region are done
    for (int k = lane; k < nsh; k += 32) sh[k] = (double)src[(long long)k * a.cs];
    __syncwarp();
    if (fmls::skip_voxel(sh, nsh)) {
      if (lane == 0) a.counts[v] = 0;
      continue;
    }
    FMLS_T(t0);
    // amplitudes (the transposed table: coalesced rows; the same FMA chain
    // over the coefficients as a row of sh2amp) and their sort keys
    for (int d = lane; d < sort_n; d += 32) {
      unsigned long long key = 0ull;  // padding: after every direction
      if (d < nd) {
        double s = 0.0;
        for (int k = 0; k < nsh; ++k) s = fma(__ldg(a.t.sh2amp_t + (long long)k * nd + d), sh[k], s);
        values[d] = s;
        key = sort_key(s, d);
      }
      keys[d] = key;
    }
    __syncwarp();
    FMLS_T(t1);
    FMLS_ACC(0, t0, t1);
    // bitonic sort, descending keys: each lane takes pairs (i, i + j)
    for (int k = 2; k <= sort_n; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int p = lane; p < (sort_n >> 1); p += 32) {
          const int i = ((p & ~(j - 1)) << 1) | (p & (j - 1));
          const unsigned long long ka = keys[i], kb = keys[i + j];
          if ((i & k) == 0 ? ka < kb : ka > kb) {
            keys[i] = kb;
            keys[i + j] = ka;
          }
        }
        __syncwarp();
      }
    }
    // keys equal above the index bits may hide magnitudes that differ in
    // their lowest 11 bits: lane 0 re-sorts such runs by the exact values
    bool tie = false;
    for (int k = lane; k + 1 < nd; k += 32) tie = tie || (keys[k] >> 11) == (keys[k + 1] >> 11);
    if (__any_sync(0xffffffffu, tie)) {
      if (lane == 0) {
        for (int k = 1; k < nd; ++k) {
          const unsigned long long x = keys[k];
          const int dx = key_dir(x);
          const double vx = fabs(values[dx]);
          int q = k;
          while (q > 0 && (keys[q - 1] >> 11) == (x >> 11)) {
            const int dy = key_dir(keys[q - 1]);
            const double vy = fabs(values[dy]);
            if (!(vx > vy || (vx == vy && dx < dy))) break;
            keys[q] = keys[q - 1];
            --q;
          }
          keys[q] = x;
        }
      }
      __syncwarp();
    }
    // the order, written over the keys it was read from (a chunk's entries
    // land below the keys later chunks read)
    for (int k0 = 0; k0 < nd; k0 += 32) {
      const int k = k0 + lane;
      const int d = k < nd ? key_dir(keys[k]) : 0;
      __syncwarp();
      if (k < nd) order[k] = (uint16_t)d;
      __syncwarp();
    }
    // the region growing (the warp) and the pending assignments (lane 0)
    FMLS_T(t2);
    FMLS_ACC(1, t1, t2);
    int nl = 0;
    bool in_smem = true;
    if (values[order[0]] > 0.0) {
      int nr = 0;
      nl = grow_warp(a.t, ws, &nr, kFmlsLobes, lane);
      FMLS_T(t3);
      FMLS_ACC(2, t2, t3);
      if (nl < 0) {  // more lobes than the shared arrays hold: lane 0 on the global slot
        in_smem = false;
        if (lane == 0) nl = fmls::grow(a.t, wg, &nr);
        nl = __shfl_sync(0xffffffffu, nl, 0);
        nr = __shfl_sync(0xffffffffu, nr, 0);
      }
      if (lane == 0) {
        if (in_smem)
          fmls::assign_pending(a.t, ws, nr);
        else
          fmls::assign_pending(a.t, wg, nr);
      }
      FMLS_T(t4);
      FMLS_ACC(3, t3, t4);
    }
    FMLS_T(t5);
    if (nl == 0) {
      if (lane == 0) a.counts[v] = 0;
      continue;
    }
    __syncwarp();
    fmls::Fixel* out = reinterpret_cast<fmls::Fixel*>(a.fixels + v * (long long)a.max_fixels * 8);
    if (in_smem) {
      // the voxel's state for the peak and finishing kernels: labels and
      // links whole, the first nl entries of the lobes' doubles
      unsigned char* gst = a.state + (size_t)c * sb;
      {
        const uint4* src = reinterpret_cast<const uint4*>(slabel);
        uint4* dst = reinterpret_cast<uint4*>(gst);
        const int nq = (int)((align16((size_t)nd) + align16((size_t)5 * kFmlsLobes)) / 16);
        for (int i = lane; i < nq; i += 32) dst[i] = src[i];
      }
      const StateView g = state_view(gst, nd);
      for (int i = lane; i < nl; i += 32) {
        g.w.max_peak[i] = ws.max_peak[i];
        g.w.integral[i] = ws.integral[i];
      }
      for (int i = lane; i < 3 * nl; i += 32) {
        g.w.mean[i] = ws.mean[i];
        g.w.peak_dir[i] = ws.peak_dir[i];
      }
      // the candidate peaks, listed with one atomic a group of 32
      for (int p0 = 0; p0 < nl; p0 += 32) {
        const int p = p0 + lane;
        const bool cand = p < nl && fmls::peak_candidate(a.t, ws, p);
        const unsigned bal = __ballot_sync(0xffffffffu, cand);
        int base = 0;
        if (lane == 0 && bal) base = atomicAdd(a.counters, __popc(bal));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (cand) a.peaks[base + __popc(bal & ((1u << lane) - 1u))] = (int)(c << kPeakShift) | p;
      }
      if (lane == 0) a.vnl[c] = nl;
      FMLS_T(t6);
      FMLS_ACC(4, t5, t6);
    } else {
      // lane 0 refines the peaks itself, in finish_lobes
      if (lane == 0) a.counts[v] = fmls::finish_lobes(a.t, wg, sh, nl, out, a.max_fixels);
    }
    __syncwarp();
  }
}

// The Newton refinements of every listed candidate peak of the round
// (SH::get_peak, SH.h:515-560), a thread a peak.  A thread takes the next
// listed peak as soon as its own has converged or run its 50 steps, so the
// lanes of a warp stay busy whatever the peaks' step counts; the taking is
// one atomic a warp for all its lanes that need a peak.  The peak's voxel's
// coefficients sit in the thread's column of shared memory (FP32, as
// given), and so do the Legendre values of each step, interpolated once
// from the table's two rows (PrecomputedAL::get) instead of at every use;
// results go to the voxel's state.
struct ShColumn {
  const float* p;
  __device__ double operator[](int k) const { return (double)p[k * kPeakThreads]; }
};
struct AlColumn {
  const double* p;
  __device__ double operator()(int l, int m) const { return p[(l * l / 4 + m) * kPeakThreads]; }
};

__global__ void __launch_bounds__(kPeakThreads) fmls_peak_kernel(const __grid_constant__ FmlsArgs a) {
  extern __shared__ __align__(16) double alcol[];  // [n_al][kPeakThreads], then the coefficients
  const int tid = threadIdx.x, lane = tid & 31;
  const int nd = a.t.ndir, nsh = a.t.nsh, n_al = a.t.n_al;
  float* shcol = reinterpret_cast<float*>(alcol + (size_t)n_al * kPeakThreads);  // [nsh][kPeakThreads]
  const size_t sb = fmls_state_bytes(nd);
  const int total = a.counters[0];
  const ShColumn sh{shcol + tid};
  int cur = -1;  // the peak this thread refines (its list entry)
  bool live = true;
  int it = 0;
  double u[3] = {0.0, 0.0, 0.0};
  for (;;) {
    const bool need = live && cur < 0;
    const unsigned nm = __ballot_sync(0xffffffffu, need);
    if (nm) {
      const int leader = __ffs(nm) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(a.counters + 1, __popc(nm));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(nm & ((1u << lane) - 1u));
        if (idx < total) {
          cur = a.peaks[idx];
          const long long c = cur >> kPeakShift;
          const int p = cur & ((1 << kPeakShift) - 1);
          const float* src = a.fod + (a.v0 + c) * a.vs;
          for (int k = 0; k < nsh; ++k) shcol[k * kPeakThreads + tid] = src[(long long)k * a.cs];
          const StateView g = state_view(a.state + (size_t)c * sb, nd);
          u[0] = g.w.peak_dir[3 * p];
          u[1] = g.w.peak_dir[3 * p + 1];
          u[2] = g.w.peak_dir[3 * p + 2];
          it = 0;
        } else {
          live = false;
        }
      }
    }
    if (!__any_sync(0xffffffffu, cur >= 0)) break;
    if (cur >= 0) {
      double val;
      const bool conv = fmls::newton_step(
          [&](double el, double az, double* dv) {
            int row;
            double f1, f2;
            fmls::al_weights(a.t, el, &row, &f1, &f2);
            for (int k = 0; k < n_al; ++k) alcol[k * kPeakThreads + tid] = fmls::al_value(a.t, row, f1, f2, k);
            fmls::derivatives_with(a.t, sh, AlColumn{alcol + tid}, el, az, dv);
          },
          u, &val);
      if (conv || ++it == fmls::kPeakSteps) {
        if (!conv) {
          u[0] = u[1] = u[2] = NAN;
          val = NAN;
        }
        const long long c = cur >> kPeakShift;
        const int p = cur & ((1 << kPeakShift) - 1);
        const StateView g = state_view(a.state + (size_t)c * sb, nd);
        g.pre_val[p] = val;
        g.pre_u[3 * p] = u[0];
        g.pre_u[3 * p + 1] = u[1];
        g.pre_u[3 * p + 2] = u[2];
        cur = -1;
      }
    }
  }
}

// fmls.cpp:258-301 for the round's voxels left by the growing kernel, a
// thread a voxel: thresholds, the nearest-peak test with the refined peaks,
// the fixels.
__global__ void __launch_bounds__(128) fmls_finish_kernel(const __grid_constant__ FmlsArgs a) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= a.nc) return;
  const int nl = a.vnl[c];
  if (nl <= 0) return;
  const int nd = a.t.ndir;
  const StateView g = state_view(a.state + (size_t)c * fmls_state_bytes(nd), nd);
  const long long v = a.v0 + c;
  fmls::Fixel* out = reinterpret_cast<fmls::Fixel*>(a.fixels + v * (long long)a.max_fixels * 8);
  a.counts[v] = fmls::finish_lobes(a.t, g.w, static_cast<const double*>(nullptr), nl, out, a.max_fixels,
                                   g.pre_val, g.pre_u);
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
  double *unit = nullptr, *weight = nullptr, *sh2amp = nullptr, *sh2amp_t = nullptr, *al = nullptr, *dsqrt = nullptr;
  int32_t *adj_off = nullptr, *adj = nullptr, *grid_off = nullptr, *grid = nullptr;
  char* scratch = nullptr;
  size_t scratch_warps = 0;
  // one round's voxel states, lobe counts, peak list and counters
  unsigned char* state = nullptr;
  int* vnl = nullptr;
  int* peaks = nullptr;
  int* counters = nullptr;
};

extern "C" void csd_fmls_destroy(csd_fmls* p) {
  if (!p) return;
  cudaFree(p->unit);
  cudaFree(p->weight);
  cudaFree(p->sh2amp);
  cudaFree(p->sh2amp_t);
  cudaFree(p->al);
  cudaFree(p->dsqrt);
  cudaFree(p->adj_off);
  cudaFree(p->adj);
  cudaFree(p->grid_off);
  cudaFree(p->grid);
  cudaFree(p->scratch);
  cudaFree(p->state);
  cudaFree(p->vnl);
  cudaFree(p->peaks);
  cudaFree(p->counters);
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
  std::vector<double> sh2amp_t((size_t)nd * c->nsh);
  for (int d = 0; d < nd; ++d)
    for (int k = 0; k < c->nsh; ++k) sh2amp_t[(size_t)k * nd + d] = c->sh2amp[(size_t)d * c->nsh + k];
  if (e == cudaSuccess) e = upload(&p->sh2amp_t, sh2amp_t.data(), sh2amp_t.size());
  if (e == cudaSuccess) e = upload(&p->al, c->al, (size_t)c->al_ndir * c->n_al);
  if (e == cudaSuccess) e = upload(&p->adj_off, c->adj_off, (size_t)nd + 1);
  if (e == cudaSuccess) e = upload(&p->adj, c->adj, (size_t)c->n_adj);
  if (e == cudaSuccess) e = upload(&p->grid_off, c->grid_off, (size_t)ncell + 1);
  if (e == cudaSuccess) e = upload(&p->grid, c->grid, (size_t)c->n_grid);
  std::vector<double> dsq((size_t)fmls::dsqrt_index(c->lmax + 1, 0), 0.0);
  for (int l = 0; l <= c->lmax; ++l)
    for (int m = 0; m <= l; ++m)
      for (int q = 0; q < 4; ++q) dsq[fmls::dsqrt_index(l, m) + q] = fmls::dsqrt_value(l, m, q);
  if (e == cudaSuccess) e = upload(&p->dsqrt, dsq.data(), dsq.size());
  if (e != cudaSuccess) {
    csd_fmls_destroy(p);
    return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_create: ") + cudaGetErrorString(e));
  }
  p->t = fmls::Tables{nd, c->lmax, c->nsh, p->unit, p->weight, p->adj_off, p->adj, p->sh2amp, c->al_ndir, c->n_al,
                      c->al_inc, p->al, c->num_az, c->num_el, c->az_begin, c->el_begin, c->az_step, c->el_step,
                      p->grid_off, p->grid, c->integral_threshold, c->peak_value_threshold, c->merge_ratio,
                      p->dsqrt, p->sh2amp_t};
  *out = p;
  return CSD_OK;
}

// Profiling hook: per-phase cycle totals of fmls_segment_kernel since the
// last reset (only in a build with -DCSD_PHASE_TIMERS; returns -5 otherwise).
extern "C" int csd_debug_fmls_cycles(unsigned long long* out, int reset) {
#ifdef CSD_PHASE_TIMERS
  if (cudaMemcpyFromSymbol(out, g_fmls_cycles, sizeof(unsigned long long) * 8) != cudaSuccess)
    return csdb200::set_error(CSD_ERR_CUDA, "csd_debug_fmls_cycles: copy failed");
  if (reset) {
    unsigned long long z[8] = {};
    cudaMemcpyToSymbol(g_fmls_cycles, z, sizeof(z));
  }
  return CSD_OK;
#else
  (void)out;
  (void)reset;
  return csdb200::set_error(CSD_ERR_UNSUPPORTED, "built without CSD_PHASE_TIMERS");
#endif
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
  const size_t slot_bytes = (align16((size_t)kSlotInts * nd * sizeof(int)) +
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
  if (!p->state) {
    e = cudaMalloc(&p->state, (size_t)kFmlsChunk * fmls_state_bytes(nd));
    if (e == cudaSuccess) e = cudaMalloc(&p->vnl, (size_t)kFmlsChunk * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&p->peaks, (size_t)kFmlsChunk * kFmlsLobes * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&p->counters, 2 * sizeof(int));
    if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
  }
  // the peak kernel: a persistent grid, its blocks' coefficient columns in shared memory
  const size_t psmem = (size_t)p->t.n_al * kPeakThreads * sizeof(double) + (size_t)nsh * kPeakThreads * sizeof(float);
  int peak_per_sm = 0;
  e = cudaFuncSetAttribute(fmls_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&peak_per_sm, fmls_peak_kernel, kPeakThreads, psmem);
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
  const unsigned peak_blocks = (unsigned)(nsm * std::max(1, peak_per_sm));
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  // rounds of kFmlsChunk voxels: growing (a warp a voxel), the peaks (a thread
  // a peak), finishing (a thread a voxel)
  for (long long v0 = 0; v0 < n; v0 += kFmlsChunk) {
    const int nc = (int)std::min<long long>(kFmlsChunk, n - v0);
    FmlsArgs a{p->t, fod, n, voxel_stride, coef_stride, mask, max_fixels, counts, fixels, p->scratch,
               (long long)slot_bytes, sort_n, v0, nc, p->state, p->vnl, p->peaks, p->counters};
    e = cudaMemsetAsync(p->counters, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) break;
    const unsigned gblocks = (unsigned)std::min<long long>(blocks, (nc + kFmlsWarps - 1) / kFmlsWarps);
    fmls_segment_kernel<<<gblocks, kFmlsWarps * 32, smem, st>>>(a);
    fmls_peak_kernel<<<peak_blocks, kPeakThreads, psmem, st>>>(a);
    fmls_finish_kernel<<<(unsigned)((nc + 127) / 128), 128, 0, st>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) break;
  }
  if (e != cudaSuccess) return csdb200::set_error(CSD_ERR_CUDA, std::string("csd_fmls_segment: ") + cudaGetErrorString(e));
  return CSD_OK;
}
