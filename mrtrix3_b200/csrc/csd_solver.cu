// libcsd_b200: kernels and C ABI of the B200-native single-shell CSD.
//
// Replaces the per-voxel ThreadedLoop of MRtrix3 `dwi2fod csd`
// (cmd/dwi2fod.cpp:275-281, core/algo/threaded_loop.h:324-362): instead of
// CPU threads taking rows of voxels under a mutex, persistent warps take
// voxels from a device work counter.  A warp that finishes a voxel (whatever
// its iteration count) immediately takes the next one, so unconverged voxels
// never hold back converged ones and volumes of uneven size share one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/csd_b200.h"
#include "csd_device.cuh"
#include "umma.cuh"
#include "shared_init.hpp"

using namespace csdb200;

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
namespace csdb200 {
extern int g_mlp_infer_kind;  // mlp.cu
extern int g_amp2sh_kind;     // amp2sh.cu
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace csdb200

#define CUDA_TRY(expr)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(CSD_ERR_CUDA, std::string(#expr " failed: ") + cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char* csd_last_error(void) { return g_err.c_str(); }

// launch-shape knobs chosen by the autotuner (0 = the built-in default)
static int g_tune_persistent_warps = 0;  // warps per block of csd_persistent_kernel
static int g_tune_solve_warps = 0;       // warps per block of csd_solve_kernel
static int g_tune_proj_blocks_per_sm = 0;
static int g_proj_kind = 0;  // projection kernel: 0 default, 1 mma.sync, 2 tcgen05 (nhr <= 320)
static int g_solve_kind = 0;  // phased solve kernel: 0 default, 1 warp per voxel, 2 / 3 groups of 16 / 8 lanes
static constexpr int kSolveDefault = 1;
static int g_set_kind = 0;    // phased set kernel: 0 default, 1 warp per voxel, 2 tiles of 64 voxels
// jump of exactly periodic two-cycles to their last call (knob 7: 0 default, 1 on, 2 off): on by default in
// the phased method (it removes ~40 near-empty passes per volume); off by default in the persistent kernel,
// where a cycling voxel only holds its own warp and the extra checks in every iteration cost more (83.8 vs
// 87.9 ms per benchmark volume)
static int g_fast_cycles = 0;
static int g_host_slabs = 0;  // host-buffer phased entry point: most slabs per call (knob 8; 0 = 8)
static int g_reuse = 0;       // later solves of warm-started voxels from their warm-set factor (knob 10: 0 default
                              // = on, 1 on, 2 off)
static int g_host_async = 0;  // host-buffer phased entry point: every slab's passes enqueued without host round
                              // trips (knob 11: 0 default = on, 1 on, 2 off: one round trip per batch of passes)
static int g_host_conc = 0;   // host-buffer phased entry point (asynchronous form): slabs computing at once (knob 13;
                              // 0 = all); slab k's compute waits for slab k - conc's, so the slabs finish one after
                              // another and their downloads overlap the later slabs' compute
static int g_asm_kind = 0;    // rank-k assembly of the phased solve (knob 12): 0 default, 1 mma.sync inside the
                              // solve kernel, 2 tcgen05 (csd_assemble_tc_kernel) ahead of it (nhr <= 320)
static constexpr int kAsmDefault = 2;
static constexpr int kSetDefault = 2;
static constexpr int kProjDefault = 2;  // tcgen05 where the table fits (nhr <= 320)


// ---------------------------------------------------------------------------
// kernels

namespace csdb200 {

template <int N>
__device__ __forceinline__ bool same_set(const uint32_t* a, const uint32_t* b, int nw) {
  bool same = true;
#pragma unroll
  for (int p = 0; p < kMaxWords; ++p)
    if (p < nw) same = same && (a[p] == b[p]);
  return same;
}

// Solve voxel v of volume V with one warp (CSD_Processor::operator(),
// cmd/dwi2fod.cpp:128-147, with CSD::set/iterate, csd.h:237-269).
template <int N>
__device__ void solve_voxel(const VolumeDesc& V, long long v, const HTab<N>& H, int nw, float cond_thr,
                            int refine, bool fast_cycles, const WarpWS<N>& w, int lane, double* slot,
                            long long* tacc = nullptr) {
  const Scheme& sc = V.sc;
  const int nhr = H.nhr;
  const bool masked = V.mask && !V.mask[v];
  const float* dwi = V.dwi + v * V.vox_stride;
  float* out = V.fod + v * V.fod_stride;
  CSD_T0(tset);
  int st = voxel_set<N>(sc, dwi, V.vol_stride, masked, w, lane);
  CSD_T1(tacc, kPhSet, tset);
  if (st != 0) {
    for (int c = lane; c < N; c += 32) out[c] = 0.f;
    if (lane == 0) {
      if (V.status) V.status[v] = (uint8_t)(st == 1 ? CSD_STATUS_MASKED : CSD_STATUS_NONFINITE);
      if (V.iters) V.iters[v] = 0;
    }
    if (V.negmask)
      for (int p = lane; p < nw; p += 32) V.negmask[v * nw + p] = 0u;
    return;
  }
  uint32_t bits[kMaxWords];
  uint32_t* old = w.old;  // warp-uniform, kept in shared memory
  uint32_t* old2 = w.old2;
  if (lane < kMaxWords) old[lane] = 0u;
  __syncwarp();
  int flags = 0, it = 0;
  bool conv = false, use_warm = V.warm != nullptr;
  for (int attempt = 0; attempt < 2; ++attempt) {
    bool have_old = false, fp32_factor = false, refined = false;
    int k = 0, rmode = refine;
    int mode_since = 0;  // every solve from this iteration on used the current rmode
    conv = false;
#pragma unroll 1
    for (it = 0; it < sc.niter; ++it) {
      if (it == 0 && use_warm) {
        // warm start: the first negative set is supplied instead of projected
#pragma unroll
        for (int p = 0; p < kMaxWords; ++p) bits[p] = (p < nw) ? __ldg(V.warm + v * nw + p) : 0u;
        if (nhr & 31) bits[nw - 1] &= (1u << (nhr & 31)) - 1u;
      } else {
        CSD_T0(tp);
        project_mask<N>(H, nw, sc.threshold, w, lane, bits);
        CSD_T1(tacc, kPhProject, tp);
        // a set that returns after one step is an FP32 two-cycle around a
        // sign change: refine every remaining solve of this voxel
        if ((rmode == 2 || rmode == 3) && it >= 2 && same_set<N>(bits, old2, nw)) {
          rmode = 1;
          mode_since = it;
        }
        if (have_old && same_set<N>(bits, old, nw)) {  // csd.h:252-253
          if (rmode == 2 && fp32_factor && !refined) {
            // refine the fixed point once, then check that it still is one
            CSD_T0(tr);
            refine_step<N>(sc, H, k, w, lane);
            CSD_T1(tacc, kPhRefine, tr);
            refined = true;
            CSD_T0(tp2);
            project_mask<N>(H, nw, sc.threshold, w, lane, bits);
            CSD_T1(tacc, kPhProject, tp2);
            if (same_set<N>(bits, old, nw)) {
              conv = true;
              ++it;
              break;
            }
            // refinement moved the set: this voxel sits close to a sign
            // change, so refine after every remaining solve
            rmode = 1;
            mode_since = it;
          } else {
            conv = true;
            ++it;
            break;
          }
        } else if (fast_cycles && it >= 2 && it >= mode_since + 2 && it + 1 < sc.niter &&
                   same_set<N>(bits, old2, nw)) {
          // a two-cycle whose both sets were last solved with the current
          // refinement mode repeats exactly (a solve depends only on its
          // set): go to the last call, whose set is this one if an even
          // number of calls remain after it, else the last solved one
          if ((sc.niter - (it + 1)) & 1) {
#pragma unroll
            for (int p = 0; p < kMaxWords; ++p)
              if (p < nw) bits[p] = old[p];
          }
          it = sc.niter - 1;
        }
      }
      CSD_T0(tl);
      k = mask_to_list(bits, nw, w.neg, lane);
      CSD_T1(tacc, kPhList, tl);
      const int fl = assemble_solve<N>(sc, H, k, w, lane, cond_thr, rmode, slot, tacc);
      flags |= fl & 0xF0;
      fp32_factor = !(fl & 0x100);
      refined = rmode == 1 && fp32_factor;
      __syncwarp();
      if (lane == 0) {
#pragma unroll
        for (int p = 0; p < kMaxWords; ++p)
          if (p < nw) {
            old2[p] = old[p];
            old[p] = bits[p];
          }
      }
      __syncwarp();
      have_old = true;
    }
    // niter exhausted: still refine the last solution
    if (!conv && rmode == 2 && fp32_factor && !refined && it > 0) refine_step<N>(sc, H, k, w, lane);
    if (conv || !use_warm || sc.niter == 0) break;
    // the warm-started iteration did not reach a fixed point: restart the
    // voxel from the plain start
    flags |= CSD_STATUS_WARM_RESTART;
    use_warm = false;
    if (lane < kMaxWords) old[lane] = 0u;
    __syncwarp();
    voxel_set<N>(sc, dwi, V.vol_stride, false, w, lane);
  }
  for (int c = lane; c < N; c += 32) out[c] = w.F[c];
  if (lane == 0) {
    const int outcome = (conv || sc.niter == 0) ? CSD_STATUS_CONVERGED : CSD_STATUS_NITER;
    if (V.status) V.status[v] = (uint8_t)(outcome | flags);
    if (V.iters) V.iters[v] = (uint8_t)(it > 255 ? 255 : it);
  }
  if (V.negmask && lane < nw) V.negmask[v * nw + lane] = old[lane];
  __syncwarp();
}

template <int N>
__global__ void __launch_bounds__(Dims<N>::THREADS, 1) csd_persistent_kernel(const __grid_constant__ SolveParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nhr = P.nhr;
  const HTab<N> H = load_htab<N>(smem, P.vol[0].sc, nhr);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  WarpWS<N> w = carve_ws<N>(smem + htab_bytes<N>(nhr) + warp * warp_ws_bytes<N>());
  double* slot = P.fp64_scratch + (size_t)(blockIdx.x * nwarps + warp) * Dims<N>::WSZ;
#ifdef CSD_PHASE_TIMERS
  long long tacc[kPhTotal + 1] = {};
  const long long tstart = clock64();
#else
  long long* tacc = nullptr;
#endif
  for (;;) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(P.queue, 1ULL);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= (unsigned long long)P.total) break;
    int vi = 0;
    while (vi + 1 < P.n_vol && (long long)g >= P.vol[vi + 1].first) ++vi;
    const VolumeDesc& V = P.vol[vi];
    solve_voxel<N>(V, (long long)g - V.first, H, P.nw, P.cond_thr, P.refine, P.fast_cycles != 0, w, lane, slot,
                   tacc);
  }
#ifdef CSD_PHASE_TIMERS
  tacc[kPhTotal] = clock64() - tstart;
  if (lane == 0)
    for (int p = 0; p <= kPhTotal; ++p) atomicAdd(&g_phase_cycles[p], (unsigned long long)tacc[p]);
#endif
}

}  // namespace csdb200

namespace csdb200 {

// ---- phased kernels behind the csd_state_* surface ------------------------
//
// The plain GPU method: one pass per CSD::iterate() over every still-active
// voxel.  csd_project_kernel evaluates HR_trans F for all active voxels as
// one dense tensor-core contraction ([voxels x nSH] x [nSH x directions],
// FP16 hi/lo split, three products, FP32 accumulation) with the sign test,
// the comparison with the previous set and the compaction fused into its
// epilogue; csd_solve_kernel then assembles and factorises (warp per voxel)
// only the voxels whose set changed.

constexpr int kProjRows = 64;       // voxels per projection tile
// Before the FP16 split each voxel's F is scaled by the power of two that
// puts its largest coefficient in [2^14, 2^15) (fp16_split_exponent), and the
// tables are HR_trans * 2^-hexp: the sign test is unchanged and a threshold
// is compared after the same exact scaling.

// status byte while iterating: low nibble 0xF, high bits = flags; 0x80 marks
// a voxel whose set cycles in FP32 (its solves are refined)
constexpr uint8_t kActive = 0x0F;
constexpr uint8_t kCycling = 0x80;

// A warp's appends to the next active list, gathered in its lanes and
// written 32 at a time with one atomic on the list's counter (every voxel of
// a pass goes through that one counter).
struct WarpAppend {
  int v = 0, n = 0;
  __device__ __forceinline__ void push(int voxel, int* list, int* counter, int lane) {
    if (lane == n) v = voxel;
    if (++n == 32) flush(list, counter, lane);
  }
  __device__ __forceinline__ void flush(int* list, int* counter, int lane) {
    if (n == 0) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(counter, n);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (lane < n) list[base + lane] = v;
    n = 0;
  }
};

// ---- factor reuse for warm-started voxels ----------------------------------
// A warm-started voxel's first solve factorises W0 = Mt_M + H[S0]^T H[S0] for
// the network's set S0 (csd.h:255-264 with S0 in place of the projected set).
// Every later set S of that voxel differs from S0 by a few directions (9 of
// 300 on average on the benchmark volume), so with C = [h_d : d in S xor S0]
// (n x r) and D = +1 for a direction S adds, -1 for one it drops,
//   W_S = W0 + C D C^T,   F = W_S^-1 b = L0^-T (y0 - U t),
// where L0 is W0's Cholesky factor, U = L0^-1 C, y0 = L0^-1 b, and t solves the
// r x r system (D + U^T U) t = U^T y0 (the Woodbury identity).  That system is
// quasi-definite -- I + U_a^T U_a > 0 on the added block, U_r^T U_r - I < 0 on
// the dropped one because W0 >= Mt_M + C_r C_r^T -- so it is eliminated on its
// diagonal without pivoting.  The iteration, its sets and its stopping rule
// are the plain method's; only the way each later W_S^-1 b is computed
// changes (r^2 n + r n^2 / 2 + n^2 operations instead of k n^2 / 2 + n^3 / 3).
#ifndef CSD_REUSE_MAXR
#define CSD_REUSE_MAXR 16
#endif
#ifndef CSD_REUSE_THREADS45
#define CSD_REUSE_THREADS45 768
#endif
constexpr int kReuseMaxR = CSD_REUSE_MAXR;  // more changed directions than this: full solve
constexpr int kReuseKS = kReuseMaxR + 1;    // row stride of [K | rhs] in shared memory (rhs in the last column)

template <int N>
struct ReuseLayout {
  static constexpr int LSZ = packoff(N + 1) + ((N + 3) / 4) * 4;  // factor rows 0..N (row N = y0), then 1/L_ii
  static constexpr int US = hr_stride(N);                         // column stride of U (odd number of float4s)
  // a warp's block, rounded to 16 bytes: the next warp's factor is read as float4s
  static constexpr int WARP_FLOATS = (LSZ + kReuseMaxR * US + kReuseMaxR * kReuseKS + 3) / 4 * 4;
  static_assert(LSZ % 4 == 0 && US % 4 == 0 && WARP_FLOATS % 4 == 0, "float4 alignment of the warp blocks");
  // threads per block (bounds the registers: U's column lives in N of them)
  static constexpr int THREADS = N <= 45 ? CSD_REUSE_THREADS45 : (N <= 66 ? 384 : 256);
};

struct StateParams {
  Scheme sc;
  int nhr, nw, n_in, use_warm, npd;
  float* Lst;           // [cap][ReuseLayout<N>::LSZ] first-solve factors of warm-started voxels, or NULL
  uint8_t* fac;         // [cap] 1 = Lst holds the factor of the voxel's warm set
  int* rest_out;        // csd_solve_reuse_kernel: the listed voxels it leaves to the full solve kernel
  int* n_rest;
  float cond_thr, thr;  // thr: the threshold (csd.h:179) in HR_trans F units
  int hexp;             // the projection tables hold HR_trans * 2^-hexp
  const __half* Hp16;   // [2][npd][HS16] projection table (hi, lo), zero rows past nhr
  const __half* Htc16;  // [2][K chunks][320 rows][8] tcgen05 projection table (hi, lo), core-matrix layout
  float* F;             // [cap][HS]
  double* b;            // [cap][N]
  uint32_t* old;        // [cap][nw] set of the last solve
  uint32_t* old2;       // [cap][nw] set of the solve before
  uint32_t* newm;       // [cap][nw] set found by the projection
  const uint32_t* warm; // [cap][nw] or NULL
  uint8_t* status;      // [cap]
  uint16_t* iters;      // [cap] iterate() calls made
  uint16_t* cyc;        // [cap] calls made when the voxel was first seen cycling
  int fast_cycles;      // jump periodic two-cycles to their last call
  const int* act_in;    // [n_in] voxel ids
  const int* n_in_dev;  // device count of act_in (overrides n_in when set)
  int* act_out;         // compacted output list
  int* n_out;
  int* err;             // set to 1 when a bounded wait times out
  unsigned long long* stats;  // [0] sum of |neg| over solves, [1] solves
  double* fp64_scratch;
  // tcgen05 assembly: W of list entries [c0, c0 + ch), row e - c0 of Wg
  float* Wg;                // [ch][packoff(N)] assembled systems
  const __half* Ptc16;      // product table (asm_shape layout)
  int pexp;                 // the product table holds HR_trans products * 2^-pexp
  int c0, ch;               // list entries of this chunk (ch = INT_MAX: all)
  // set() inputs
  const float* dwi;
  long long vox_stride, vol_stride;
  const uint8_t* mask;
};

// CSD::set for every voxel (csd.h:237-243); voxels that are masked out or
// hold a non-finite sample are finished immediately with F = 0.
template <int N>
__global__ void __launch_bounds__(256) csd_state_set_kernel(const __grid_constant__ StateParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpWS<N> w = carve_ws<N>(smem + warp * warp_ws_bytes<N>());
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
  const long long nwt = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long v = gw; v < P.n_in; v += nwt) {
    const bool masked = P.mask && !P.mask[v];
    const int st = voxel_set<N>(P.sc, P.dwi + v * P.vox_stride, P.vol_stride, masked, w, lane);
    float* F = P.F + v * Dims<N>::HS;
    for (int c = lane; c < Dims<N>::HS; c += 32) F[c] = st ? 0.f : w.F[c];
    for (int c = lane; c < N; c += 32) P.b[v * N + c] = st ? 0.0 : w.b[c];
    for (int p = lane; p < P.nw; p += 32) {
      P.old[v * P.nw + p] = 0u;
      P.old2[v * P.nw + p] = 0u;
    }
    if (lane == 0) {
      P.iters[v] = 0;
      if (st) {
        P.status[v] = (uint8_t)(st == 1 ? CSD_STATUS_MASKED : CSD_STATUS_NONFINITE);
      } else if (P.sc.niter == 0) {
        P.status[v] = CSD_STATUS_CONVERGED;
      } else {
        P.status[v] = kActive;
        P.act_out[atomicAdd(P.n_out, 1)] = (int)v;
      }
    }
  }
}

// set() over tiles of 64 voxels (csd.h:237-243 with dwi2fod.cpp:156-173):
// the block stages the tile's selected, clamped DW samples and the scheme's
// rconv^T / M tables in shared memory, then each thread forms F = rconv S
// and b = M^T S for 4 voxels x ceil(N/16) coefficients in registers, with
// the summation order of voxel_set (two accumulators over the samples in
// steps of 4, the remainder on the first), so the results are the same bit
// for bit.  Status, iteration counters and the active list follow
// csd_state_set_kernel; the list is compacted with one atomic per warp.
constexpr int kSetTile = 64;

__host__ __device__ constexpr int set_tile_lds(int ndw) { return ((ndw + 3) & ~3) + 1; }

__host__ __device__ constexpr size_t set_tile_smem(int ndw, int ninit, int n) {
  return (size_t)ndw * (ninit + n) * 4 + (size_t)kSetTile * set_tile_lds(ndw) * 4 + kSetTile * 4;
}

template <int N>
__global__ void __launch_bounds__(256) csd_state_set_tile_kernel(const __grid_constant__ StateParams P) {
  constexpr int JC = (N + 15) / 16;
  extern __shared__ __align__(16) unsigned char smem[];
  const int ndw = P.sc.ndw, ninit = P.sc.ninit;
  const int lds = set_tile_lds(ndw);
  float* rT = reinterpret_cast<float*>(smem);  // [ndw][ninit]
  float* Mt = rT + ndw * ninit;                 // [ndw][N]
  float* S = Mt + ndw * N;                      // [kSetTile][lds]
  int* flag = reinterpret_cast<int*>(S + kSetTile * lds);  // 0 ok, 1 masked, 3 non-finite
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < ndw * ninit; i += blockDim.x) rT[i] = __ldg(P.sc.rconvT + i);
  for (int i = tid; i < ndw * N; i += blockDim.x) Mt[i] = __ldg(P.sc.M32 + i);
  const int vg = tid >> 4, cg = tid & 15;
  const int nd4 = ndw & ~3;
  const long long ntiles = (P.n_in + kSetTile - 1) / kSetTile;
  // the selected volumes' offsets of this lane's sample slots (up to 3 a lane)
  constexpr int kSetChunks = 3;
  long long off[kSetChunks];
#pragma unroll
  for (int c = 0; c < kSetChunks; ++c) {
    const int t = lane + 32 * c;
    off[c] = t < ndw ? (long long)__ldg(P.sc.dwis + t) * P.vol_stride : 0;
  }
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const long long v0 = tile * kSetTile;
    __syncthreads();
    if (ndw <= 32 * kSetChunks) {
      // 1. samples: warp w stages voxels w, w + 8, ..., w + 56, every load
      // issued before any is used (lane j < 8 reads voxel j's mask byte)
      bool in = false;
      if (lane < kSetTile / 8) {
        const long long v = v0 + warp + 8 * lane;
        in = v < P.n_in && !(P.mask && !P.mask[v]);
      }
      const unsigned inm = __ballot_sync(0xffffffffu, in);
      float x[kSetTile / 8][kSetChunks];
#pragma unroll
      for (int j = 0; j < kSetTile / 8; ++j) {
        const float* d = P.dwi + (v0 + warp + 8 * j) * P.vox_stride;
#pragma unroll
        for (int c = 0; c < kSetChunks; ++c)
          x[j][c] = (((inm >> j) & 1u) && lane + 32 * c < ndw) ? __ldg(d + off[c]) : 0.f;
      }
#pragma unroll
      for (int j = 0; j < kSetTile / 8; ++j) {
        const int r = warp + 8 * j;
        bool bad = false;
#pragma unroll
        for (int c = 0; c < kSetChunks; ++c) {
          const int t = lane + 32 * c;
          if (t < ndw) {
            bad = bad || !isfinite(x[j][c]);
            S[r * lds + t] = x[j][c] < 0.f ? 0.f : x[j][c];
          }
        }
        const bool anybad = __any_sync(0xffffffffu, bad);
        if (lane == 0) flag[r] = ((inm >> j) & 1u) ? (anybad ? 3 : 0) : 1;
      }
    } else {
    // 1. samples: warp w stages voxels w, w + 8, ...
    for (int r = warp; r < kSetTile; r += 8) {
      const long long v = v0 + r;
      int f = 1;
      if (v < P.n_in && !(P.mask && !P.mask[v])) {
        const float* d = P.dwi + v * P.vox_stride;
        bool bad = false;
        for (int t = lane; t < ndw; t += 32) {
          const float x = __ldg(d + (long long)__ldg(P.sc.dwis + t) * P.vol_stride);
          if (!isfinite(x)) bad = true;
          S[r * lds + t] = x < 0.f ? 0.f : x;
        }
        f = __any_sync(0xffffffffu, bad) ? 3 : 0;
      }
      if (lane == 0) flag[r] = f;
    }
    }
    __syncthreads();  // the flags are complete before anyone reads them (the vote's
                      // predicate is evaluated before its own barrier)
    // a tile with no voxel to solve (outside the mask) only writes zeros
    const bool any = __syncthreads_or(tid < kSetTile && flag[tid] == 0);
    // 2. F and b for voxels 4 vg .. 4 vg + 3, coefficients cg + 16 j
    float f0[4][JC], f1[4][JC], b0[4][JC], b1[4][JC];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int j = 0; j < JC; ++j) f0[a][j] = f1[a][j] = b0[a][j] = b1[a][j] = 0.f;
    const float* S0 = S + (4 * vg) * lds;
    int t = any ? 0 : ndw;
    for (; t < nd4; t += 4) {
#pragma unroll
      for (int tt = 0; tt < 4; ++tt) {
        float sv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) sv[a] = S0[a * lds + t + tt];
#pragma unroll
        for (int j = 0; j < JC; ++j) {
          const int c = cg + 16 * j;
          if (c < N) {
            const float m = Mt[(t + tt) * N + c];
            const float r = c < ninit ? rT[(t + tt) * ninit + c] : 0.f;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
              if (tt & 1) {
                if (c < ninit) f1[a][j] = fmaf(r, sv[a], f1[a][j]);
                b1[a][j] = fmaf(m, sv[a], b1[a][j]);
              } else {
                if (c < ninit) f0[a][j] = fmaf(r, sv[a], f0[a][j]);
                b0[a][j] = fmaf(m, sv[a], b0[a][j]);
              }
            }
          }
        }
      }
    }
    for (; t < ndw; ++t) {
      float sv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) sv[a] = S0[a * lds + t];
#pragma unroll
      for (int j = 0; j < JC; ++j) {
        const int c = cg + 16 * j;
        if (c < N) {
          const float m = Mt[t * N + c];
          const float r = c < ninit ? rT[t * ninit + c] : 0.f;
#pragma unroll
          for (int a = 0; a < 4; ++a) {
            if (c < ninit) f0[a][j] = fmaf(r, sv[a], f0[a][j]);
            b0[a][j] = fmaf(m, sv[a], b0[a][j]);
          }
        }
      }
    }
    // (a voxel that is not solved -- masked or non-finite -- keeps no F, b or
    // sets: csd_state_fod writes its zeros from the status)
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int r = 4 * vg + a;
      const long long v = v0 + r;
      if (v >= P.n_in || flag[r] != 0) continue;
      float* F = P.F + v * Dims<N>::HS;
#pragma unroll
      for (int j = 0; j < JC; ++j) {
        const int c = cg + 16 * j;
        if (c < N) {
          F[c] = f0[a][j] + f1[a][j];
          P.b[v * N + c] = (double)(b0[a][j] + b1[a][j]);
        }
      }
      for (int c = N + cg; c < Dims<N>::HS; c += 16) F[c] = 0.f;
    }
    // 3. counters, sets and the active list
    for (int i = tid; i < kSetTile * P.nw; i += blockDim.x) {
      const long long v = v0 + i / P.nw;
      if (v < P.n_in && flag[i / P.nw] == 0) {
        P.old[v0 * P.nw + i] = 0u;
        P.old2[v0 * P.nw + i] = 0u;
      }
    }
    if (warp < kSetTile / 32) {
      const int r = 32 * warp + lane;
      const long long v = v0 + r;
      bool act = false;
      if (v < P.n_in) {
        const int f = flag[r];
        P.iters[v] = 0;
        if (f) {
          P.status[v] = (uint8_t)(f == 1 ? CSD_STATUS_MASKED : CSD_STATUS_NONFINITE);
        } else if (P.sc.niter == 0) {
          P.status[v] = CSD_STATUS_CONVERGED;
        } else {
          P.status[v] = kActive;
          act = true;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, act);
      int base = 0;
      if (lane == 0 && bal) base = atomicAdd(P.n_out, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (act) P.act_out[base + __popc(bal & ((1u << lane) - 1u))] = (int)v;
    }
  }
}

// Two-cycles (csd.h:246-253 iterated to niter).  A voxel whose new set
// equals the one before last (`back`) is flagged cycling (st |= kCycling,
// cyc = calls made) and from then on solves with one refinement step.  Once
// both sets of the cycle have been solved with refinement (two calls after
// the flag), the iteration is exactly periodic: a solve is a deterministic
// function of its set, so F and the sets alternate until niter.  The voxel
// then jumps to its last call: solve now with the set the niter-th call
// would use (this one if niter - calls is even, else the last solved one,
// in `old`) and finish with niter calls -- the same FOD, set and count as
// running every call.  Returns 0 (no jump), 1 (jump, this set), 2 (jump,
// the last solved set); updates st / cyc when the cycle is first seen.
__device__ __forceinline__ int cycle_jump(const StateParams& P, long long v, int it, bool warm, bool back,
                                          uint8_t& st) {
  if (warm || it < 2 || !back) return 0;
  if (!(st & kCycling)) {
    st |= kCycling;
    if (P.cyc) P.cyc[v] = (uint16_t)it;
    return 0;
  }
  if (!P.fast_cycles || !P.cyc || it < (int)P.cyc[v] + 2 || it + 1 >= P.sc.niter) return 0;
  return ((P.sc.niter - (it + 1)) & 1) ? 2 : 1;
}

// Whether voxel v's solve in this pass goes through its stored warm-set
// factor.  Warp-collective (every lane returns the same answer); lane p < nw
// receives word p of the added / dropped directions, r their total.  The
// reuse and the full solve kernels evaluate it on the same state, the reuse
// kernel first: a voxel it cannot finish has fac cleared and so falls to the
// full kernel in the same pass.
__device__ __forceinline__ bool reuse_route(const StateParams& P, long long v, int lane, uint32_t& add,
                                            uint32_t& rem, int& r) {
  add = rem = 0u;
  r = 0;
  if (!P.fac || !P.warm || !P.use_warm) return false;
  if (!P.fac[v] || P.iters[v] < 2 || (P.status[v] & kCycling)) return false;
  if (lane < P.nw) {
    const uint32_t nb = P.newm[v * P.nw + lane];
    uint32_t wb = P.warm[v * P.nw + lane];
    if (lane == P.nw - 1 && (P.nhr & 31)) wb &= (1u << (P.nhr & 31)) - 1u;
    add = nb & ~wb;
    rem = wb & ~nb;
  }
  r = __reduce_add_sync(0xffffffffu, __popc(add) + __popc(rem));
  return r <= kReuseMaxR;
}

// Later solves of warm-started voxels from the stored factor of their warm
// set (see ReuseLayout): warp per voxel.  Lane j < r carries column j of C
// (the FP32 constraint row of the j-th changed direction, added ones first)
// through the forward substitution with L0; the pairs of K = D + U^T U are
// spread over the lanes; [K | U^T y0] is eliminated by the lanes (one row
// each); then x = y0 - U t and F = L0^-T x.  Bookkeeping of sets, counts and
// the next active list is the full solve kernel's.  (Packing several voxels
// into one warp's lanes fills the idle lanes of the forward substitution but
// needs their factors in shared memory together: at 7 warps an SM it ran
// 1.6x slower than this form at 16.)
template <int N>
__global__ void __launch_bounds__(ReuseLayout<N>::THREADS, 1)
    csd_solve_reuse_kernel(const __grid_constant__ StateParams P) {
  using RL = ReuseLayout<N>;
  constexpr int HS = Dims<N>::HS;
  constexpr int CQ = Dims<N>::CQ;
  constexpr int NQ = Dims<N>::NQ;
  extern __shared__ __align__(16) float rsm[];
  const int nwarps = blockDim.x >> 5;
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  if ((long long)blockIdx.x * nwarps >= n_in) return;  // the grid is an upper bound
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* Lb = rsm + (size_t)warp * RL::WARP_FLOATS;  // factor rows 0..N (row N = y0), then 1/L_ii
  float* Ub = Lb + RL::LSZ;                          // [kReuseMaxR][US] columns of U
  float* Kb = Ub + kReuseMaxR * RL::US;              // [kReuseMaxR][kReuseKS] rows of [K | rhs]
  const float* rd = Lb + packoff(N + 1);
  const float* y0 = Lb + packoff(N);
  int* dl = reinterpret_cast<int*>(Kb);              // changed directions (before K is formed)
  unsigned long long n_solved = 0, sum_r = 0;  // work counters (stats[2], [3]), added once per warp
  WarpAppend app;
  for (int e = blockIdx.x * nwarps + warp; e < n_in; e += gridDim.x * nwarps) {
    const long long v = P.act_in[e];
    // the stored factor into shared memory (coalesced 16-byte copies), issued
    // before the routing test so that both round trips overlap (the host
    // launches this kernel only on passes where nearly every listed voxel
    // has a factor)
    {
      const float4* src = reinterpret_cast<const float4*>(P.Lst + (size_t)v * RL::LSZ);
      float4* dst = reinterpret_cast<float4*>(Lb);
      for (int i = lane; i < RL::LSZ / 4; i += 32) dst[i] = __ldcs(src + i);
    }
    uint32_t add, rem;
    int r;
    if (!reuse_route(P, v, lane, add, rem, r)) {
      if (lane == 0 && P.rest_out) P.rest_out[atomicAdd(P.n_rest, 1)] = (int)v;
      __syncwarp();
      continue;
    }
    // the changed directions in order: added ones, then dropped ones.  Lane
    // p < nw owns word p: an exclusive scan of the words' counts gives its
    // place, then it writes its words' set bits.
    int na = 0;
    {
      const int ca = __popc(add), cr = __popc(rem);
      int xa = ca, xr = cr;  // inclusive scans over the lanes
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const int ya = __shfl_up_sync(0xffffffffu, xa, o), yr = __shfl_up_sync(0xffffffffu, xr, o);
        if (lane >= o) {
          xa += ya;
          xr += yr;
        }
      }
      na = __shfl_sync(0xffffffffu, xa, 15);  // words live in lanes 0..15 (kMaxWords)
      int pa = xa - ca, pr = na + xr - cr;
      for (uint32_t w = add; w; w &= w - 1u) dl[pa++] = 32 * lane + __ffs(w) - 1;
      for (uint32_t w = rem; w; w &= w - 1u) dl[pr++] = 32 * lane + __ffs(w) - 1;
    }
    __syncwarp();
    // U = L0^-1 C in shared memory (column j of U at Ub + j US), blocked by
    // 8 rows: the r column lanes solve a block's diagonal part, then every
    // lane takes one of the rows below it and subtracts the block's
    // contribution from that row of every column.  (One column a lane over
    // all 45 rows left 23 of 32 lanes idle for most of the kernel.)
    {
      constexpr int Q4 = RL::US / 4;
      for (int it = lane; it < r * Q4; it += 32) {
        const int j = it / Q4, q = it - j * Q4;
        const int dj = dl[j];
        reinterpret_cast<float4*>(Ub + j * RL::US)[q] =
            4 * q < HS ? __ldg(reinterpret_cast<const float4*>(P.sc.H32 + (size_t)dj * HS) + q)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    }
    __syncwarp();
#pragma unroll
    for (int i0 = 0; i0 < N; i0 += 8) {
      constexpr int BW = 8;
      const int nb = N - i0 < BW ? N - i0 : BW;  // rows of this block (compile-time after unrolling)
      if (lane < r) {
        float* uc = Ub + lane * RL::US + i0;
        float v[BW];
#pragma unroll
        for (int t = 0; t < BW; ++t) {
          if (t < nb) {
            const float* Li = Lb + packoff(i0 + t) + i0;
            float s0 = uc[t], s1 = 0.f;
#pragma unroll
            for (int e = 0; e < t; e += 2) {
              s0 = fmaf(-Li[e], v[e], s0);
              if (e + 1 < t) s1 = fmaf(-Li[e + 1], v[e + 1], s1);
            }
            v[t] = (s0 + s1) * rd[i0 + t];
          }
        }
#pragma unroll
        for (int t = 0; t < BW; ++t)
          if (t < nb) uc[t] = v[t];
      }
      __syncwarp();
      if (i0 + BW < N) {
        // rows i0 + 8 .. N - 1: lane l takes rows i0 + 8 + l (+ 32)
#pragma unroll
        for (int rb = i0 + BW; rb < N; rb += 32) {
          const int i = rb + lane;
          if (i < N) {
            const float4 la = *reinterpret_cast<const float4*>(Lb + packoff(i) + i0);
            const float4 lb = *reinterpret_cast<const float4*>(Lb + packoff(i) + i0 + 4);
            for (int j = 0; j < r; ++j) {
              const float* uc = Ub + j * RL::US;
              const float4 ua = *reinterpret_cast<const float4*>(uc + i0);
              const float4 ub = *reinterpret_cast<const float4*>(uc + i0 + 4);
              float s0 = uc[i], s1 = 0.f;
              s0 = fmaf(-la.x, ua.x, s0);
              s1 = fmaf(-la.y, ua.y, s1);
              s0 = fmaf(-la.z, ua.z, s0);
              s1 = fmaf(-la.w, ua.w, s1);
              s0 = fmaf(-lb.x, ub.x, s0);
              s1 = fmaf(-lb.y, ub.y, s1);
              s0 = fmaf(-lb.z, ub.z, s0);
              s1 = fmaf(-lb.w, ub.w, s1);
              Ub[j * RL::US + i] = s0 + s1;
            }
          }
        }
      }
      __syncwarp();
    }
    // rhs_j = u_j . y0
    float rhs0 = 0.f, rhs1 = 0.f;
    if (lane < r) {
      const float4* uc = reinterpret_cast<const float4*>(Ub + lane * RL::US);
      const float4* y4 = reinterpret_cast<const float4*>(y0);
#pragma unroll
      for (int q = 0; q < NQ; ++q) {  // only rows < N: y0's padding is not cleared
        const float4 x = uc[q], y = y4[q];
        rhs0 = fmaf(x.x, y.x, rhs0);
        if (4 * q + 1 < N) rhs1 = fmaf(x.y, y.y, rhs1);
        if (4 * q + 2 < N) rhs0 = fmaf(x.z, y.z, rhs0);
        if (4 * q + 3 < N) rhs1 = fmaf(x.w, y.w, rhs1);
      }
    }
    __syncwarp();
    // K = D + U^T U: pair p = j (j + 1) / 2 + i, i <= j, spread over the lanes
    const int npair = r * (r + 1) / 2;
    for (int p = lane; p < npair; p += 32) {
      int j = (int)((sqrtf(8.f * (float)p + 1.f) - 1.f) * 0.5f);
      while ((j + 1) * (j + 2) / 2 <= p) ++j;
      while (j * (j + 1) / 2 > p) --j;
      const int i = p - j * (j + 1) / 2;
      const float4* ci = reinterpret_cast<const float4*>(Ub + i * RL::US);
      const float4* cj = reinterpret_cast<const float4*>(Ub + j * RL::US);
      float a0 = 0.f, a1 = 0.f;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        const float4 x = ci[q], y = cj[q];
        a0 = fmaf(x.x, y.x, a0);
        a1 = fmaf(x.y, y.y, a1);
        a0 = fmaf(x.z, y.z, a0);
        a1 = fmaf(x.w, y.w, a1);
      }
      const float kij = a0 + a1 + (i == j ? (i < na ? 1.f : -1.f) : 0.f);
      Kb[i * kReuseKS + j] = kij;
      Kb[j * kReuseKS + i] = kij;
    }
    if (lane < r) Kb[lane * kReuseKS + kReuseMaxR] = rhs0 + rhs1;
    __syncwarp();
    // Gauss-Jordan elimination of [K | rhs] on the diagonal (quasi-definite)
    bool ok = true;
    for (int p = 0; p < r; ++p) {
      const float piv = Kb[p * kReuseKS + p];
      ok = ok && isfinite(piv) && piv != 0.f;
      const float rpiv = __frcp_rn(piv);
      if (ok && lane < r && lane != p) {
        const float f = Kb[lane * kReuseKS + p] * rpiv;
        for (int c = p; c < r; ++c) Kb[lane * kReuseKS + c] = fmaf(-f, Kb[p * kReuseKS + c], Kb[lane * kReuseKS + c]);
        Kb[lane * kReuseKS + kReuseMaxR] =
            fmaf(-f, Kb[p * kReuseKS + kReuseMaxR], Kb[lane * kReuseKS + kReuseMaxR]);
      }
      __syncwarp();
    }
    const float t = (ok && lane < r) ? Kb[lane * kReuseKS + kReuseMaxR] / Kb[lane * kReuseKS + lane] : 0.f;
    if (!__all_sync(0xffffffffu, ok && isfinite(t))) {
      // leave this voxel to the full solve kernel of the same pass
      if (lane == 0) {
        P.fac[v] = 0;
        if (P.rest_out) P.rest_out[atomicAdd(P.n_rest, 1)] = (int)v;
      }
      __syncwarp();
      continue;
    }
    // x = y0 - U t, then F = L0^-T x
    float x[CQ];
#pragma unroll
    for (int q = 0; q < CQ; ++q) {
      const int i = lane + 32 * q;
      x[q] = i < N ? y0[i] : 0.f;
    }
    for (int j = 0; j < r; ++j) {
      const float tj = __shfl_sync(0xffffffffu, t, j);
#pragma unroll
      for (int q = 0; q < CQ; ++q) {
        const int i = lane + 32 * q;
        if (i < N) x[q] = fmaf(-Ub[j * RL::US + i], tj, x[q]);
      }
    }
    chol_back_f32<N>(Lb, rd, x, lane);
#pragma unroll
    for (int q = 0; q < CQ; ++q) {
      const int i = lane + 32 * q;
      if (i < N) P.F[v * HS + i] = x[q];
    }
    if (lane < P.nw) {
      P.old2[v * P.nw + lane] = P.old[v * P.nw + lane];
      P.old[v * P.nw + lane] = P.newm[v * P.nw + lane];
    }
    sum_r += (unsigned long long)r;
    ++n_solved;
    {
      const uint8_t flags = (uint8_t)(P.status[v] & 0x70);
      const bool last = P.iters[v] >= P.sc.niter;
      __syncwarp();
      if (lane == 0) P.status[v] = last ? (uint8_t)(CSD_STATUS_NITER | flags) : (uint8_t)(kActive | flags);
      if (!last) app.push((int)v, P.act_out, P.n_out, lane);
    }
    __syncwarp();
  }
  app.flush(P.act_out, P.n_out, lane);
  if (lane == 0 && P.stats && n_solved) {
    atomicAdd(P.stats + 2, n_solved);
    atomicAdd(P.stats + 3, sum_r);
  }
}

// Projection pass: tiles of 64 active voxels.  Warp w computes rows
// 16 (w & 3) .. +15 against half (w >> 2) of the directions with mma.sync
// m16n8k16 (F hi/lo from shared memory as A, the direction table as B, both
// K-major, loaded by ldmatrix); the epilogue sets one bit per negative
// amplitude in a shared bitmap, then each voxel's bitmap is compared with
// its previous set (csd.h:246-253): converged voxels finish, the others go
// to the solve list.
template <int N>
__global__ void __launch_bounds__(256) csd_project_kernel(const __grid_constant__ StateParams P) {
  using D = Dims<N>;
  constexpr int KS = D::NRB;                 // k16 steps over the coefficients
  extern __shared__ __align__(16) unsigned char smem[];
  const int npd = P.npd;                     // directions padded to a multiple of 32
  __half* Hh = reinterpret_cast<__half*>(smem);
  __half* Hl = Hh + npd * D::HS16;
  __half* Fh = Hl + npd * D::HS16;
  __half* Fl = Fh + kProjRows * D::HS16;
  uint32_t* bm = reinterpret_cast<uint32_t*>(Fl + kProjRows * D::HS16);  // [64][kMaxWords]
  float* rowscale = reinterpret_cast<float*>(bm + kProjRows * kMaxWords);  // [64] F scale of each row
  float* rowthr = rowscale + kProjRows;                                     // [64] threshold in scaled units
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  if ((long long)blockIdx.x * kProjRows >= n_in) return;  // the grid is an upper bound
  {
    const uint4* src = reinterpret_cast<const uint4*>(P.Hp16);
    uint4* dst = reinterpret_cast<uint4*>(Hh);
    for (int i = threadIdx.x; i < 2 * npd * D::HS16 / 8; i += blockDim.x) dst[i] = __ldg(src + i);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int mrow = 16 * (warp & 3);
  const int half = warp >> 2;
  constexpr int tpw = 20;                    // n8 tiles per warp: half of a 320-direction chunk
  const int ntiles = (n_in + kProjRows - 1) / kProjRows;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int e0 = tile * kProjRows;
    __syncthreads();
    // per-row power-of-two scale of F (warp w: rows w, w + 8, ...)
    for (int r = warp; r < kProjRows; r += 8) {
      float mx = 0.f;
      if (e0 + r < n_in)
        for (int c = lane; c < N; c += 32) mx = fmaxf(mx, fabsf(P.F[(long long)P.act_in[e0 + r] * D::HS + c]));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) {
        const float sc = pow2f(-fp16_split_exponent(mx));
        rowscale[r] = sc;
        rowthr[r] = P.thr * sc * pow2f(-P.hexp);
      }
    }
    __syncthreads();
    // F rows -> scaled FP16 hi / lo
    for (int i = threadIdx.x; i < kProjRows * D::HS16; i += blockDim.x) {
      const int r = i / D::HS16, c = i - r * D::HS16;
      float f = 0.f;
      if (e0 + r < n_in && c < N) f = P.F[(long long)P.act_in[e0 + r] * D::HS + c] * rowscale[r];
      const __half h = __float2half_rn(f);
      Fh[i] = h;
      Fl[i] = __float2half_rn(f - __half2float(h));
    }
    for (int i = threadIdx.x; i < kProjRows * kMaxWords; i += blockDim.x) bm[i] = 0u;
    __syncthreads();
    for (int c0 = 0; c0 < npd; c0 += 320) {
    float acc[20][4];
#pragma unroll
    for (int t = 0; t < 20; ++t)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[t][e] = 0.f;
#pragma unroll
    for (int ks = 0; ks < KS; ++ks) {
      uint32_t ah[4], al[4];
      ldsm4(ah, Fh + (mrow + (lane & 15)) * D::HS16 + 16 * ks + (lane >> 4) * 8);
      ldsm4(al, Fl + (mrow + (lane & 15)) * D::HS16 + 16 * ks + (lane >> 4) * 8);
#pragma unroll
      for (int t = 0; t < 20; t += 2) {
        {
          const int nb = c0 + 8 * (half * tpw + t);
          const int noff = (lane & 7) + ((lane >> 4) << 3), koff = ((lane >> 3) & 1) * 8;
          uint32_t bh[4], bl[4];
          ldsm4(bh, Hh + (nb + noff) * D::HS16 + 16 * ks + koff);
          ldsm4(bl, Hl + (nb + noff) * D::HS16 + 16 * ks + koff);
          mma_f16(acc[t], ah, bh[0], bh[1]);
          mma_f16(acc[t], ah, bl[0], bl[1]);
          mma_f16(acc[t], al, bh[0], bh[1]);
          mma_f16(acc[t + 1], ah, bh[2], bh[3]);
          mma_f16(acc[t + 1], ah, bl[2], bl[3]);
          mma_f16(acc[t + 1], al, bh[2], bh[3]);
        }
      }
    }
    const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int t = 0; t < 20; ++t) {
      {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int r = mrow + gid + 8 * (e >> 1);
          const int c = c0 + 8 * (half * tpw + t) + 2 * tig + (e & 1);
          if (c < P.nhr && acc[t][e] < rowthr[r]) atomicOr(&bm[r * kMaxWords + (c >> 5)], 1u << (c & 31));
        }
      }
    }
    }
    __syncthreads();
    // per-voxel decision: warp w handles rows w, w + 8, ...
    for (int r = warp; r < kProjRows; r += 8) {
      if (e0 + r >= n_in) break;
      const long long v = P.act_in[e0 + r];
      const int it = P.iters[v];
      const bool warm = it == 0 && P.use_warm && P.warm;
      uint32_t bits = 0u;
      if (lane < P.nw) {
        bits = warm ? P.warm[v * P.nw + lane] : bm[r * kMaxWords + lane];
        if (warm && lane == P.nw - 1 && (P.nhr & 31)) bits &= (1u << (P.nhr & 31)) - 1u;
      }
      const bool same = __all_sync(0xffffffffu, lane >= P.nw || bits == P.old[v * P.nw + lane]);
      const bool back = __all_sync(0xffffffffu, lane >= P.nw || bits == P.old2[v * P.nw + lane]);
      const bool conv = !warm && it > 0 && same;
      uint8_t st = P.status[v];
      const int ff = cycle_jump(P, v, it, warm, back, st);
      if (!conv && lane < P.nw) P.newm[v * P.nw + lane] = ff == 2 ? P.old[v * P.nw + lane] : bits;
      if (lane == 0) {
        P.iters[v] = (uint16_t)(ff ? P.sc.niter : it + 1);
        if (conv) {
          P.status[v] = (uint8_t)(CSD_STATUS_CONVERGED | (st & 0x70));
        } else {
          P.status[v] = st;
          P.act_out[atomicAdd(P.n_out, 1)] = (int)v;
        }
      }
    }
  }
}

// First pass of a warm-started run: every active voxel's first set is the
// supplied one (csd.h:246-250 is skipped for it, as the projection kernels
// do at it == 0), so no amplitudes are needed: copy the set (its last word
// masked to nhr directions), count the call, and list every voxel for its
// first solve -- the state the projection kernels leave at it == 0.
__global__ void __launch_bounds__(256) csd_warm_first_pass_kernel(const __grid_constant__ StateParams P) {
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  const int lane = threadIdx.x & 31;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long e0 = (long long)blockIdx.x * blockDim.x; e0 < n_in; e0 += stride) {
    const long long e = e0 + threadIdx.x;
    const bool act = e < n_in;
    long long v = 0;
    if (act) {
      v = P.act_in[e];
      for (int w = 0; w < P.nw; ++w) {
        uint32_t b = P.warm[v * P.nw + w];
        if (w == P.nw - 1 && (P.nhr & 31)) b &= (1u << (P.nhr & 31)) - 1u;
        P.newm[v * P.nw + w] = b;
      }
      P.iters[v] = 1;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, act);
    int base = 0;
    if (lane == 0 && bal) base = atomicAdd(P.n_out, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (act) P.act_out[base + __popc(bal & ((1u << lane) - 1u))] = (int)v;
  }
}

// ---- tcgen05 projection (sm_100a): the same pass as csd_project_kernel on
// the 5th-generation tensor cores.  A tile of 128 active voxels is the
// M=128 operand (F, split into FP16 hi/lo, scaled by 2^8), the 320-row
// direction table the N operand (two N=160 instructions), K = 16 per
// instruction; D accumulates hi*hi + hi*lo + lo*hi in FP32 in tensor memory
// (320 of 512 allocated columns).  Operands sit in shared memory in the
// canonical K-major, non-swizzled layout: 8-row x 16-byte core matrices,
// row groups SBO = 128 B apart, K chunks LBO apart.  One elected thread
// issues the instructions and commits them to an mbarrier; every thread
// then reads its own voxel's row of D (tcgen05.ld 32x32b), packs the sign
// bits, and makes the convergence decision itself.  Waits are bounded: on
// time-out the kernel raises an error flag, frees its tensor memory and
// returns.

constexpr int kTcRows = 128;          // voxels per tile (M)
constexpr int kTcDirs = 320;          // directions (N, two instructions of 160)

template <int N>
__global__ void __launch_bounds__(128, 1) csd_project_tc_kernel(const __grid_constant__ StateParams P) {
  using D = Dims<N>;
  constexpr int KC = 2 * D::NRB;                     // 8-half K chunks
  constexpr int A_BYTES = KC * (kTcRows / 8) * 128;  // one of hi / lo
  constexpr int B_BYTES = KC * (kTcDirs / 8) * 128;
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned char* sBh = smem;
  unsigned char* sBl = sBh + B_BYTES;
  unsigned char* sAh = sBl + B_BYTES;
  unsigned char* sAl = sAh + A_BYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sAl + A_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  const int ntiles = (n_in + kTcRows - 1) / kTcRows;
  if ((int)blockIdx.x >= ntiles) return;  // the grid is an upper bound; before any allocation
  // direction table (host-prepared in the core-matrix layout), once per block
  {
    const uint4* src = reinterpret_cast<const uint4*>(P.Htc16);
    uint4* dst = reinterpret_cast<uint4*>(sBh);
    for (int i = tid; i < 2 * B_BYTES / 16; i += blockDim.x) dst[i] = __ldg(src + i);
  }
  const uint32_t mbar_a = static_cast<uint32_t>(__cvta_generic_to_shared(mbar));
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar_a));
  }
  if (warp == 0) {
    const uint32_t slot = static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot));
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(slot));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_f16(kTcRows, kTcDirs / 2);
  const uint32_t aH = static_cast<uint32_t>(__cvta_generic_to_shared(sAh));
  const uint32_t aL = static_cast<uint32_t>(__cvta_generic_to_shared(sAl));
  const uint32_t bH = static_cast<uint32_t>(__cvta_generic_to_shared(sBh));
  const uint32_t bL = static_cast<uint32_t>(__cvta_generic_to_shared(sBl));
  constexpr uint32_t A_LBO = (kTcRows / 8) * 128, B_LBO = (kTcDirs / 8) * 128;
  uint32_t phase = 0;
  bool failed = false;
  for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
    const int e0 = tile * kTcRows;
    float thr_v = 0.f;  // this row's threshold in the scaled units of its amplitudes
    // this thread's voxel row -> scaled FP16 hi / lo chunks in the core-matrix layout
    {
      const int r = tid;
      float f[KC * 8];
#pragma unroll
      for (int c = 0; c < KC * 8; ++c) f[c] = 0.f;
      if (e0 + r < n_in) {
        const float4* src = reinterpret_cast<const float4*>(P.F + (long long)P.act_in[e0 + r] * D::HS);
#pragma unroll
        for (int q = 0; q < (KC * 8) / 4; ++q) {
          if (4 * q < D::HS) {
            const float4 x = src[q];
            f[4 * q] = 4 * q < N ? x.x : 0.f;
            f[4 * q + 1] = 4 * q + 1 < N ? x.y : 0.f;
            f[4 * q + 2] = 4 * q + 2 < N ? x.z : 0.f;
            f[4 * q + 3] = 4 * q + 3 < N ? x.w : 0.f;
          }
        }
      }
      float mx = 0.f;
#pragma unroll
      for (int c = 0; c < KC * 8; ++c) mx = fmaxf(mx, fabsf(f[c]));
      const float fscale = pow2f(-fp16_split_exponent(mx));
      thr_v = P.thr * fscale * pow2f(-P.hexp);
#pragma unroll
      for (int kc = 0; kc < KC; ++kc) {
        __align__(16) __half hi[8], lo[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const float v = f[8 * kc + e] * fscale;
          hi[e] = __float2half_rn(v);
          lo[e] = __float2half_rn(v - __half2float(hi[e]));
        }
        const int off = kc * A_LBO + (r >> 3) * 128 + (r & 7) * 16;
        *reinterpret_cast<uint4*>(sAh + off) = *reinterpret_cast<const uint4*>(hi);
        *reinterpret_cast<uint4*>(sAl + off) = *reinterpret_cast<const uint4*>(lo);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    if (tid == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const uint32_t dcol = tmem + (uint32_t)(h * (kTcDirs / 2));
        const uint32_t boff = (uint32_t)(h * (kTcDirs / 16)) * 128;  // 20 row groups per half
#pragma unroll
        for (int ks = 0; ks < D::NRB; ++ks) {
          const uint32_t ak = (uint32_t)(2 * ks) * A_LBO, bk = (uint32_t)(2 * ks) * B_LBO + boff;
          const uint64_t dAh = umma_smem_desc(aH + ak, A_LBO, 128), dAl = umma_smem_desc(aL + ak, A_LBO, 128);
          const uint64_t dBh = umma_smem_desc(bH + bk, B_LBO, 128), dBl = umma_smem_desc(bL + bk, B_LBO, 128);
          const uint64_t pa[3] = {dAh, dAh, dAl}, pb[3] = {dBh, dBl, dBh};
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            const uint32_t acc = (ks > 0 || p > 0) ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred q;\n\t"
                "setp.ne.b32 q, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, q;\n\t}\n"
                :
                : "r"(dcol), "l"(pa[p]), "l"(pb[p]), "r"(idesc), "r"(acc), "r"(0u));
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar_a));
    }
    const int ok = mbar_wait(mbar_a, phase) ? 1 : 0;
    phase ^= 1u;
    if (!__syncthreads_and(ok)) {
      // give the tensor core a second bounded chance to drain before the
      // tensor memory is freed, then report the time-out
      mbar_wait(mbar_a, phase ^ 1u);
      if (tid == 0) atomicExch(P.err, 1);
      failed = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
    // this thread's row of D: sign bits of its 300 amplitudes
    uint32_t words[kTcDirs / 32];
#pragma unroll
    for (int w = 0; w < kTcDirs / 32; ++w) words[w] = 0u;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
    for (int j = 0; j < kTcDirs / 16; ++j) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(lane_addr + (uint32_t)(16 * j)));
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::);
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int c = 16 * j + e;
        if (c < P.nhr && __uint_as_float(v[e]) < thr_v) words[c >> 5] |= 1u << (c & 31);
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::);
    // per-voxel decision (csd.h:246-253), one thread per voxel
    const int r = tid;
    bool append = false;
    long long v = 0;
    if (e0 + r < n_in) {
      v = P.act_in[e0 + r];
      const int it = P.iters[v];
      const bool warm = it == 0 && P.use_warm && P.warm;
      bool same = true, back = true;
      for (int w = 0; w < P.nw; ++w) {
        uint32_t b = words[w < kTcDirs / 32 ? w : 0];
        if (warm) {
          b = P.warm[v * P.nw + w];
          if (w == P.nw - 1 && (P.nhr & 31)) b &= (1u << (P.nhr & 31)) - 1u;
        }
        words[w < kTcDirs / 32 ? w : 0] = b;
        same = same && b == P.old[v * P.nw + w];
        back = back && b == P.old2[v * P.nw + w];
      }
      const bool conv = !warm && it > 0 && same;
      uint8_t st = P.status[v];
      const int ff = cycle_jump(P, v, it, warm, back, st);
      P.iters[v] = (uint16_t)(ff ? P.sc.niter : it + 1);
      if (conv) {
        P.status[v] = (uint8_t)(CSD_STATUS_CONVERGED | (st & 0x70));
      } else {
        for (int w = 0; w < P.nw; ++w)
          P.newm[v * P.nw + w] = ff == 2 ? P.old[v * P.nw + w] : words[w < kTcDirs / 32 ? w : 0];
        P.status[v] = st;
        append = true;
      }
    }
    // the solve list, one atomic per warp (a single counter takes every append)
    {
      const unsigned bal = __ballot_sync(0xffffffffu, append);
      int base = 0;
      if ((tid & 31) == 0 && bal) base = atomicAdd(P.n_out, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (append) P.act_out[base + __popc(bal & ((1u << (tid & 31)) - 1u))] = (int)v;
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::);
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
}

// ---- tcgen05 rank-k assembly (sm_100a): W = Mt_M + H[neg]^T H[neg]
// (csd.h:255-262) for a tile of 128 listed voxels at once, as the dense
// product W[v][c] = Mt_M[c] + sum_d mask[v][d] P[d][c], with c = packoff(i)
// + j the packed position of W(i, j) and P[d][c] = h_d[i] h_d[j].  The mask
// is exact in FP16 (0 / 1), P is split into FP16 hi + lo (22 significant
// bits), so two products per instruction pair accumulate in FP32 in tensor
// memory: the rank-k update of every voxel of the tile in one pass over the
// directions.  Roles (192 threads): warps 0-3 turn each voxel's set bits
// into its row of the M=128 operand (one thread a voxel) and read the
// accumulators back (tcgen05.ld, the warp's quarter of the lanes), adding
// Mt_M and storing W to global memory for csd_solve_kernel<N, true>; warp 4
// streams the product table through kAsmStages shared-memory stages (bulk copies
// completing on mbarriers); warp 5 issues the MMAs (N = NC columns a chunk,
// K = 16 an instruction) into two tensor-memory buffers, so one chunk's
// read-back overlaps the next chunk's products.  Every wait is bounded; a
// time-out raises the error flag, and every role still reaches the final
// barrier before the tensor memory is freed.
constexpr int kAsmRows = 128;                    // voxels per tile (M)
constexpr int kAsmK = 320;                       // directions (K), nhr <= 320
#ifndef CSD_ASM_SLAB_K
#define CSD_ASM_SLAB_K 64
#endif
#ifndef CSD_ASM_STAGES
#define CSD_ASM_STAGES 2
#endif
// The product table streams through kAsmStages shared-memory stages of
// kAsmSlabK directions; while the MMAs read one stage the others are in
// flight.  Two stages of 64, four of 32 and eight of 16 directions measure
// the same (2.52 / 2.53 / 2.61 ms of assembly a benchmark step, outputs
// bit-identical): the copies in flight do not bound the kernel.
constexpr int kAsmSlabK = CSD_ASM_SLAB_K;        // directions per stage
constexpr int kAsmSlabs = kAsmK / kAsmSlabK;     // stages per chunk
constexpr int kAsmStages = CSD_ASM_STAGES;       // stages in shared memory
static_assert(kAsmK % kAsmSlabK == 0 && kAsmSlabK % 16 == 0 && kAsmStages >= 2 && kAsmStages <= 8, "stages");
constexpr int kAsmABytes = (kAsmK / 8) * kAsmRows * 16;

struct AsmShape {
  int wsz, nch, nc;   // packed W floats; column chunks of nc (a multiple of 16, <= 256)
};
__host__ __device__ constexpr AsmShape asm_shape(int n) {
  return AsmShape{packoff(n), (packoff(n) + 255) / 256,
                  (((packoff(n) + (packoff(n) + 255) / 256 - 1) / ((packoff(n) + 255) / 256)) + 15) / 16 * 16};
}
__host__ __device__ constexpr int asm_stage_bytes(int n) { return 2 * (kAsmSlabK / 8) * asm_shape(n).nc * 16; }
__host__ __device__ constexpr int asm_smem_bytes(int n) { return kAsmABytes + kAsmStages * asm_stage_bytes(n) + 256; }

__device__ __forceinline__ void mbar_arrive1(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}

template <int N>
__global__ void __launch_bounds__(192, 1) csd_assemble_tc_kernel(const __grid_constant__ StateParams P) {
  constexpr AsmShape S = asm_shape(N);
  constexpr int NC = S.nc, NCH = S.nch, WSZ = S.wsz;
  constexpr int STAGE = asm_stage_bytes(N);
  constexpr uint32_t A_LBO = (kAsmRows / 8) * 128, B_LBO = NC * 16;
  static_assert(2 * NC <= 512 && NC % 16 == 0 && NC >= 16 && NC <= 256, "chunk shape");
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sA = smem;
  unsigned char* sB = smem + kAsmABytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(sB + kAsmStages * STAGE);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kAsmStages + 6);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  const int end = min(n_in, P.c0 + P.ch);
  const int ntiles = end > P.c0 ? (end - P.c0 + kAsmRows - 1) / kAsmRows : 0;
  if ((int)blockIdx.x >= ntiles) return;  // the grid is an upper bound; before any allocation
  const uint32_t bar0 = static_cast<uint32_t>(__cvta_generic_to_shared(bars));
  // barriers: b_full[kAsmStages], b_empty[kAsmStages], acc_full[2], acc_empty[2], a_full, done
  constexpr uint32_t NS = kAsmStages;
  auto b_full = [&](int i) { return bar0 + 8u * (uint32_t)i; };
  auto b_empty = [&](int i) { return bar0 + 8u * (NS + (uint32_t)i); };
  auto acc_full = [&](int i) { return bar0 + 8u * (2 * NS + (uint32_t)i); };
  auto acc_empty = [&](int i) { return bar0 + 8u * (2 * NS + 2 + (uint32_t)i); };
  const uint32_t a_full = bar0 + 8u * (2 * NS + 4), done = bar0 + 8u * (2 * NS + 5);
  if (tid == 0) {
    for (int i = 0; i < kAsmStages; ++i) {
      mbar_init(b_full(i), 1);
      mbar_init(b_empty(i), 1);
    }
    for (int i = 0; i < 2; ++i) {
      mbar_init(acc_full(i), 1);
      mbar_init(acc_empty(i), kAsmRows);
    }
    mbar_init(a_full, kAsmRows);
    mbar_init(done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
  }
  if (warp == 0) tmem_alloc(static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot)), 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  bool failed = false;
  if (warp == 4) {
    // producer: the product table, chunk by chunk, slab by slab, for every tile
    if (lane == 0) {
      const unsigned char* src = reinterpret_cast<const unsigned char*>(P.Ptc16);
      const uint32_t sB0 = static_cast<uint32_t>(__cvta_generic_to_shared(sB));
      int it = 0;
      for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x)
        for (int ch = 0; ch < NCH && !failed; ++ch)
          for (int sl = 0; sl < kAsmSlabs; ++sl, ++it) {
            const int st = it % kAsmStages;
            const uint32_t ph = (uint32_t)(it / kAsmStages) & 1u;
            if (!mbar_wait(b_empty(st), ph ^ 1u)) {
              failed = true;
              break;
            }
            mbar_arrive_expect_tx(b_full(st), (uint32_t)STAGE);
            bulk_copy_g2s(sB0 + (uint32_t)(st * STAGE), src + (size_t)(ch * kAsmSlabs + sl) * STAGE, (uint32_t)STAGE,
                          b_full(st));
          }
      if (failed) atomicExch(P.err, 1);
    }
  } else if (warp == 5) {
    // MMA issuer
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_f16(kAsmRows, NC);
      const uint32_t aS = static_cast<uint32_t>(__cvta_generic_to_shared(sA));
      const uint32_t bS = static_cast<uint32_t>(__cvta_generic_to_shared(sB));
      int it = 0, ac = 0, tc = 0;
      for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x, ++tc) {
        if (!mbar_wait(a_full, (uint32_t)tc & 1u)) {
          failed = true;
          break;
        }
        tc_fence_after();
        for (int ch = 0; ch < NCH && !failed; ++ch, ++ac) {
          const int buf = ac & 1;
          if (!mbar_wait(acc_empty(buf), (((uint32_t)ac >> 1) & 1u) ^ 1u)) {
            failed = true;
            break;
          }
          tc_fence_after();
          const uint32_t dcol = tmem + (uint32_t)(buf * NC);
          for (int sl = 0; sl < kAsmSlabs; ++sl, ++it) {
            const int st = it % kAsmStages;
            if (!mbar_wait(b_full(st), (uint32_t)(it / kAsmStages) & 1u)) {
              failed = true;
              break;
            }
            tc_fence_after();
            const uint32_t bh = bS + (uint32_t)(st * STAGE), bl = bh + (uint32_t)(STAGE / 2);
#pragma unroll
            for (int ks = 0; ks < kAsmSlabK / 16; ++ks) {
              const uint32_t ka = (uint32_t)(2 * (sl * (kAsmSlabK / 16) + ks)) * A_LBO;
              const uint32_t kb = (uint32_t)(2 * ks) * B_LBO;
              const uint64_t da = umma_smem_desc(aS + ka, A_LBO, 128);
              umma_f16_ss(dcol, da, umma_smem_desc(bh + kb, B_LBO, 128), idesc, (sl > 0 || ks > 0) ? 1u : 0u);
              umma_f16_ss(dcol, da, umma_smem_desc(bl + kb, B_LBO, 128), idesc, 1u);
            }
            umma_commit(b_empty(st));  // the stage is free once these products are done
          }
          if (failed) break;
          umma_commit(acc_full(buf));  // the chunk's accumulators (and every earlier product) are done
        }
      }
      if (failed) atomicExch(P.err, 1);
      umma_commit(done);  // arrives once every product this thread issued has finished
    }
  } else {
    // warps 0-3: one voxel a thread -- its operand row, then its accumulators
    const int r = tid;
    const float ps = pow2f(P.pexp);
    const uint32_t lane_base = tmem + ((uint32_t)(32 * warp) << 16);
    int ac = 0;
    for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
      const int e = P.c0 + tile * kAsmRows + r;
      const bool live = e < end;
      {
        uint32_t words[kAsmK / 32];
        const long long v = live ? (long long)P.act_in[e] : 0;
#pragma unroll
        for (int w = 0; w < kAsmK / 32; ++w) words[w] = (live && w < P.nw) ? P.newm[v * P.nw + w] : 0u;
#pragma unroll
        for (int kc = 0; kc < kAsmK / 8; ++kc) {
          const uint32_t byte = (words[kc >> 2] >> (8 * (kc & 3))) & 0xFFu;
          uint32_t q[4];
#pragma unroll
          for (int t = 0; t < 4; ++t)
            q[t] = (((byte >> (2 * t)) & 1u) ? 0x3C00u : 0u) | (((byte >> (2 * t + 1)) & 1u) ? 0x3C000000u : 0u);
          *reinterpret_cast<uint4*>(sA + kc * A_LBO + (r >> 3) * 128 + (r & 7) * 16) = make_uint4(q[0], q[1], q[2], q[3]);
        }
      }
      fence_async_smem();
      mbar_arrive1(a_full);
      float* dst = P.Wg + (size_t)(e - P.c0) * WSZ;
      for (int ch = 0; ch < NCH; ++ch, ++ac) {
        const int buf = ac & 1;
        const int ok = mbar_wait(acc_full(buf), ((uint32_t)ac >> 1) & 1u) ? 1 : 0;
        if (!__all_sync(0xffffffffu, ok)) {
          failed = true;
          break;
        }
        tc_fence_after();
#pragma unroll 1
        for (int j = 0; j < NC / 16; ++j) {
          uint32_t x[16];
          tmem_ld16(lane_base + (uint32_t)(buf * NC + 16 * j), x);
          tmem_ld_wait();
          const int c = ch * NC + 16 * j;
          if (live && c < WSZ) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              if (c + 4 * q < WSZ) {
                const float4 m = __ldg(reinterpret_cast<const float4*>(P.sc.MtMp + c + 4 * q));
                float4 o;
                o.x = fmaf(__uint_as_float(x[4 * q]), ps, m.x);
                o.y = fmaf(__uint_as_float(x[4 * q + 1]), ps, m.y);
                o.z = fmaf(__uint_as_float(x[4 * q + 2]), ps, m.z);
                o.w = fmaf(__uint_as_float(x[4 * q + 3]), ps, m.w);
                __stcg(reinterpret_cast<float4*>(dst + c + 4 * q), o);
              }
            }
          }
        }
        tc_fence_before();
        mbar_arrive1(acc_empty(buf));
      }
      if (failed) {
        if (tid == 0) atomicExch(P.err, 1);
        break;
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    // no product may still be writing the tensor memory when it is freed (bounded)
    mbar_wait(done, 0u);
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// Threads per block of csd_solve_kernel<N, true> (systems assembled by
// csd_assemble_tc_kernel): no constraint tables and no assembly registers,
// so more warps fit an SM.
template <int N>
struct PreSolveThreads {
#ifdef CSD_PRE_THREADS45
  static constexpr int value = N <= 45 ? CSD_PRE_THREADS45 : Dims<N>::THREADS;
#else
  static constexpr int value = N <= 45 ? 1024 : Dims<N>::THREADS;
#endif
};

// Solve pass: warp per voxel of the solve list (csd.h:255-266).  PRE: the
// list entries [c0, c0 + ch) whose systems csd_assemble_tc_kernel left in
// Wg (row e - c0); otherwise every entry, assembled here (mma.sync).
template <int N, bool PRE = false>
__global__ void __launch_bounds__(PRE ? PreSolveThreads<N>::value : Dims<N>::SOLVE_THREADS, 1)
    csd_solve_kernel(const __grid_constant__ StateParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int HS = Dims<N>::HS;
  const int nwarps = blockDim.x >> 5;
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  const int e0 = PRE ? P.c0 : 0;
  const int end = PRE ? min(n_in, P.c0 + P.ch) : n_in;
  if ((long long)e0 + (long long)blockIdx.x * nwarps >= end) return;  // the grid is an upper bound
  HTab<N> H;
  if constexpr (PRE) {
    // only the refinement of cycling voxels reads the tables: from global memory
    H.h32 = P.sc.H32;
    H.hh = P.sc.H16;
    H.hl = P.sc.H16 + (size_t)(P.nhr + 1) * Dims<N>::HS16;
    H.nhr = P.nhr;
    H.use32 = Dims<N>::KEEP32;
    H.hs = P.sc.hscale;
  } else {
    H = load_htab<N>(smem, P.sc, P.nhr, false);
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpWS<N> w = carve_ws<N>(smem + (PRE ? 0 : htab_bytes<N>(P.nhr, false)) + warp * warp_ws_bytes<N>());
  double* slot = P.fp64_scratch + (size_t)(blockIdx.x * nwarps + warp) * Dims<N>::WSZ;
  const int gw = blockIdx.x * nwarps + warp, nwt = gridDim.x * nwarps;
#ifdef CSD_PHASE_TIMERS
  long long tacc[kPhTotal + 1] = {};
  const long long tstart = clock64();
#else
  long long* tacc = nullptr;
#endif
  unsigned long long sum_k = 0, n_solved = 0;  // work counters, added once per warp
  WarpAppend app;
  for (int e = e0 + gw; e < end; e += nwt) {
    CSD_T0(tl);
    const long long v = P.act_in[e];
    {
      uint32_t a_, r_;
      int nr_;
      if (reuse_route(P, v, lane, a_, r_, nr_)) continue;  // solved by csd_solve_reuse_kernel
    }
    if constexpr (PRE) {
      const float4* src = reinterpret_cast<const float4*>(P.Wg + (size_t)(e - e0) * Dims<N>::WSZ);
      float4* dst = reinterpret_cast<float4*>(w.W);
      for (int i = lane; i < Dims<N>::WSZ / 4; i += 32) dst[i] = __ldcs(src + i);
    }
    for (int c = lane; c < N; c += 32) w.b[c] = P.b[v * N + c];
    for (int c = lane; c < HS; c += 32) w.F[c] = 0.f;
    uint32_t bits[kMaxWords];
#pragma unroll
    for (int p = 0; p < kMaxWords; ++p) bits[p] = (p < P.nw) ? P.newm[v * P.nw + p] : 0u;
    __syncwarp();
    const uint8_t st = P.status[v];
    const int k = mask_to_list(bits, P.nw, w.neg, lane);
    sum_k += (unsigned long long)k;
    ++n_solved;
    CSD_T1(tacc, kPhList, tl);
    const int fl_all =
        assemble_solve<N, true, PRE>(P.sc, H, k, w, lane, P.cond_thr, (st & kCycling) ? 1 : 0, slot, tacc);
    const int fl = fl_all & 0x70;
    CSD_T0(tw);
    if (P.Lst && P.use_warm && P.warm && P.iters[v] == 1) {
      // first solve of a warm-started voxel: keep the FP32 factor of its warm
      // set (rows 0..N, row N = L^-1 b, then 1/L_ii) for its later solves
      const bool keep = !(fl_all & 0x100);
      if (keep) {
        constexpr int LSZ = ReuseLayout<N>::LSZ, WQ = packoff(N + 1) / 4;
        float4* dst = reinterpret_cast<float4*>(P.Lst + (size_t)v * LSZ);
        const float4* W4 = reinterpret_cast<const float4*>(w.W);
        const float4* R4 = reinterpret_cast<const float4*>(w.rdiag);
        for (int i = lane; i < LSZ / 4; i += 32) dst[i] = i < WQ ? W4[i] : R4[i - WQ];
      }
      if (lane == 0) P.fac[v] = keep ? 1 : 0;
    }
    for (int c = lane; c < N; c += 32) P.F[v * HS + c] = w.F[c];
    if (lane < P.nw) {
      P.old2[v * P.nw + lane] = P.old[v * P.nw + lane];
      P.old[v * P.nw + lane] = P.newm[v * P.nw + lane];
    }
    {
      const uint8_t flags = (uint8_t)((st & 0xF0) | fl);
      const bool last = P.iters[v] >= P.sc.niter;
      if (lane == 0) P.status[v] = last ? (uint8_t)(CSD_STATUS_NITER | (flags & 0x70)) : (uint8_t)(kActive | flags);
      if (!last) app.push((int)v, P.act_out, P.n_out, lane);
    }
    CSD_T1(tacc, kPhSet, tw);
  }
  app.flush(P.act_out, P.n_out, lane);
  if (lane == 0 && P.stats && n_solved) {
    atomicAdd(P.stats, sum_k);
    atomicAdd(P.stats + 1, n_solved);
  }
#ifdef CSD_PHASE_TIMERS
  tacc[kPhTotal] = clock64() - tstart;
  if (lane == 0)
    for (int p = 0; p <= kPhTotal; ++p) atomicAdd(&g_phase_cycles[p], (unsigned long long)tacc[p]);
#endif
}

// Solve pass with G lanes per voxel: each warp takes 32 / G voxels of the
// solve list, assembles them one after another (warp-wide tensor-core
// rank-k, as csd_solve_kernel), factorises and back-substitutes all of them
// at once (one group of G lanes per voxel), then finishes them one by one
// (FP64 fallback, refinement of cycling voxels, stores).  The arithmetic of
// every voxel is the sequence csd_solve_kernel performs, so the outputs are
// bit-identical; the grouping cuts the instructions per voxel of the
// factorisation and substitution, where a whole warp on one 45 x 45 system
// leaves most lanes idle on the short rows of the late column blocks.
template <int G>
struct GroupSolveThreads {
  static constexpr int value = G == 16 ? 416 : 224;  // 13 / 7 warps: what fits beside the tables
};

template <int N, int G>
__global__ void __launch_bounds__(GroupSolveThreads<G>::value, 1)
    csd_solve_group_kernel(const __grid_constant__ StateParams P) {
  constexpr int V = 32 / G;
  constexpr int CQG = GroupDims<N, G>::CQG;
  using Lw = GroupWSLayout<N, V>;
  constexpr int HS = Dims<N>::HS;
  extern __shared__ __align__(16) unsigned char smem[];
  const int nwarps = blockDim.x >> 5;
  const int n_in = P.n_in_dev ? *P.n_in_dev : P.n_in;
  if ((long long)blockIdx.x * nwarps * V >= n_in) return;  // the grid is an upper bound
  const HTab<N> H = load_htab<N>(smem, P.sc, P.nhr, false);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = lane / G, sl = lane % G;
  unsigned char* base = smem + htab_bytes<N>(P.nhr, false) + warp * Lw::WARP;
  double* slot64 = P.fp64_scratch + (size_t)(blockIdx.x * nwarps + warp) * Dims<N>::WSZ;
  const WarpWS<N> mine = group_slot_ws<N, V>(base, grp);
  const long long stride = (long long)gridDim.x * nwarps * V;
  unsigned long long sum_k = 0, n_solved = 0;  // work counters, added once per warp
  for (long long e0 = ((long long)blockIdx.x * nwarps + warp) * V; e0 < n_in; e0 += stride) {
    // 1. assembly of each voxel's system (+ its right-hand side as row N);
    // a voxel solved from its warm-set factor (csd_solve_reuse_kernel) leaves
    // its slot idle
    unsigned idle = 0u;
#pragma unroll 1
    for (int g = 0; g < V; ++g) {
      if (e0 + g >= n_in) break;
      const WarpWS<N> w = group_slot_ws<N, V>(base, g);
      const long long v = P.act_in[e0 + g];
      {
        uint32_t a_, r_;
        int nr_;
        if (reuse_route(P, v, lane, a_, r_, nr_)) {
          idle |= 1u << g;
          continue;
        }
      }
      for (int c = lane; c < N; c += 32) w.b[c] = P.b[v * N + c];
      for (int c = lane; c < HS; c += 32) w.F[c] = 0.f;
      uint32_t bits[kMaxWords];
#pragma unroll
      for (int p = 0; p < kMaxWords; ++p) bits[p] = (p < P.nw) ? P.newm[v * P.nw + p] : 0u;
      __syncwarp();
      const int k = mask_to_list(bits, P.nw, w.neg, lane);
      sum_k += (unsigned long long)k;
      ++n_solved;
      assemble<N, true>(H, P.sc.MtMp, k, w, lane);
      float* bN = w.W + packoff(N);
      for (int c = lane; c < packoff(N + 1) - packoff(N); c += 32) bN[c] = c < N ? (float)w.b[c] : 0.f;
      __syncwarp();
    }
    // 2. factorisation (forward solve fused) + back substitution, all voxels
    float dmin, dmax;
    const bool okl = cholesky_group_f32<N, G>(mine.W, mine.rdiag, sl, dmin, dmax);
    const float cond = okl ? (dmax / dmin) * (dmax / dmin) : 3.0e38f;
    const bool goodl = okl && (cond <= P.cond_thr);
    const unsigned good = __ballot_sync(0xffffffffu, goodl);
    float x[CQG];
#pragma unroll
    for (int q = 0; q < CQG; ++q) {
      const int i = sl + G * q;
      x[q] = i < N ? mine.W[packoff(N) + i] : 0.f;
    }
    chol_back_group_f32<N, G>(mine.W, mine.rdiag, x, sl);
    if (goodl) {
#pragma unroll
      for (int q = 0; q < CQG; ++q) {
        const int i = sl + G * q;
        if (i < N) mine.F[i] = x[q];
      }
    }
    __syncwarp();
    // 3. per voxel: FP64 fallback / refinement, stores, next active list
#pragma unroll 1
    for (int g = 0; g < V; ++g) {
      if (e0 + g >= n_in) break;
      if ((idle >> g) & 1u) continue;
      const WarpWS<N> w = group_slot_ws<N, V>(base, g);
      const long long v = P.act_in[e0 + g];
      const uint8_t st = P.status[v];
      const bool ok = (good >> (g * G)) & 1u;
      if (P.Lst && P.use_warm && P.warm && P.iters[v] == 1) {
        // first solve of a warm-started voxel: keep its FP32 factor, as csd_solve_kernel does
        if (ok) {
          constexpr int LSZ = ReuseLayout<N>::LSZ, WQ = packoff(N + 1) / 4;
          float4* dst = reinterpret_cast<float4*>(P.Lst + (size_t)v * LSZ);
          const float4* W4 = reinterpret_cast<const float4*>(w.W);
          const float4* R4 = reinterpret_cast<const float4*>(w.rdiag);
          for (int i = lane; i < LSZ / 4; i += 32) dst[i] = i < WQ ? W4[i] : R4[i - WQ];
        }
        if (lane == 0) P.fac[v] = ok ? 1 : 0;
      }
      int fl = 0;
      if (!ok || (st & kCycling)) {
        // the shared list holds the last voxel's set: rebuild this one's
        uint32_t bits[kMaxWords];
#pragma unroll
        for (int p = 0; p < kMaxWords; ++p) bits[p] = (p < P.nw) ? P.newm[v * P.nw + p] : 0u;
        const int k = mask_to_list(bits, P.nw, w.neg, lane);
        if (!ok)
          fl = 0x10 | (solve_fp64<N>(P.sc, k, w, slot64, lane) ? 0 : 0x20);
        else
          refine_step<N>(P.sc, H, k, w, lane);
      }
      for (int c = lane; c < N; c += 32) P.F[v * HS + c] = w.F[c];
      if (lane < P.nw) {
        P.old2[v * P.nw + lane] = P.old[v * P.nw + lane];
        P.old[v * P.nw + lane] = P.newm[v * P.nw + lane];
      }
      if (lane == 0) {
        const uint8_t flags = (uint8_t)((st & 0xF0) | fl);
        if (P.iters[v] >= P.sc.niter) {
          P.status[v] = (uint8_t)(CSD_STATUS_NITER | (flags & 0x70));
        } else {
          P.status[v] = (uint8_t)(kActive | flags);
          P.act_out[atomicAdd(P.n_out, 1)] = (int)v;
        }
      }
      __syncwarp();
    }
  }
  if (lane == 0 && P.stats && n_solved) {
    atomicAdd(P.stats, sum_k);
    atomicAdd(P.stats + 1, n_solved);
  }
}

// FP64 check of every finished voxel's last solve: the residual
// r = b - (Mt_M + H_S^T H_S) F of its final set S (csd.h:255-264) in FP64 with
// the FP64 tables, and rho = max|r| / max|b|.  A voxel with rho above `tol`
// has its system re-assembled, factorised and solved in FP64 (its status
// gains CSD_STATUS_FP64).  Warp per voxel: the lanes first take the
// directions of S (a_d = h_d . F), then the coefficients
// (sum_d a_d h_d + Mt_M F).  Up to lmax 8 the block keeps HR_trans and Mt_M
// (FP64) in shared memory.  ctr[0] += voxels checked, ctr[1] += re-solved.
template <int N>
struct CheckLayout {
  static constexpr bool STAGE = N <= 45;  // FP64 tables in shared memory
  static constexpr int WARP = warp_ws_bytes<N>() + (kMaxHR + Dims<N>::HS) * 8;
  static constexpr int WARPS = STAGE ? 8 : 4;
  static size_t table_bytes(int nhr) { return STAGE ? ((size_t)nhr * N + (size_t)N * N) * 8 : 0; }
};

template <int N>
__global__ void __launch_bounds__(256) csd_state_check_kernel(const __grid_constant__ StateParams P, long long n,
                                                               double tol, unsigned long long* ctr) {
  using CL = CheckLayout<N>;
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double* H = P.sc.H64;      // [nhr][N]
  const double* MtM = P.sc.MtM64;  // [N][N]
  size_t tb = 0;
  if (CL::STAGE) {
    double* hs = reinterpret_cast<double*>(smem);
    const int nh = P.nhr * N, nm = N * N;
    for (int i = threadIdx.x; i < nh; i += blockDim.x) hs[i] = __ldg(P.sc.H64 + i);
    for (int i = threadIdx.x; i < nm; i += blockDim.x) hs[nh + i] = __ldg(P.sc.MtM64 + i);
    H = hs;
    MtM = hs + nh;
    tb = ((size_t)(nh + nm) * 8 + 15) & ~(size_t)15;
    __syncthreads();
  }
  unsigned char* mine = smem + tb + warp * CL::WARP;
  WarpWS<N> w = carve_ws<N>(mine);
  double* ad = reinterpret_cast<double*>(mine + warp_ws_bytes<N>());  // a_d of the set's directions
  double* Fd = ad + kMaxHR;                                            // F in FP64
  double* slot = P.fp64_scratch + (size_t)(blockIdx.x * (blockDim.x >> 5) + warp) * Dims<N>::WSZ;
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
  const long long nwt = (long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long checked = 0, resolved = 0;
  for (long long v = gw; v < n; v += nwt) {
    const uint8_t st = P.status[v];
    const int outcome = st & 0x0F;
    if (outcome != CSD_STATUS_CONVERGED && outcome != CSD_STATUS_NITER) continue;
    for (int c = lane; c < N; c += 32) {
      Fd[c] = (double)P.F[v * Dims<N>::HS + c];
      w.b[c] = P.b[v * N + c];
    }
    uint32_t bits[kMaxWords];
#pragma unroll
    for (int p = 0; p < kMaxWords; ++p) bits[p] = (p < P.nw) ? P.old[v * P.nw + p] : 0u;
    const int k = mask_to_list(bits, P.nw, w.neg, lane);
    __syncwarp();
    for (int q = lane; q < k; q += 32) {
      const double* h = H + (int)w.neg[q] * N;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
#pragma unroll
      for (int i = 0; i < N; i += 4) {
        a0 = fma(h[i], Fd[i], a0);
        if (i + 1 < N) a1 = fma(h[i + 1], Fd[i + 1], a1);
        if (i + 2 < N) a2 = fma(h[i + 2], Fd[i + 2], a2);
        if (i + 3 < N) a3 = fma(h[i + 3], Fd[i + 3], a3);
      }
      ad[q] = (a0 + a1) + (a2 + a3);
    }
    __syncwarp();
    double rmax = 0.0, bmax = 0.0;
#pragma unroll
    for (int c = 0; c < Dims<N>::CQ; ++c) {
      const int i = lane + 32 * c;
      if (i < N) {
        double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
        int q = 0;
        for (; q + 3 < k; q += 4) {
          u0 = fma(ad[q], H[(int)w.neg[q] * N + i], u0);
          u1 = fma(ad[q + 1], H[(int)w.neg[q + 1] * N + i], u1);
          u2 = fma(ad[q + 2], H[(int)w.neg[q + 2] * N + i], u2);
          u3 = fma(ad[q + 3], H[(int)w.neg[q + 3] * N + i], u3);
        }
        for (; q < k; ++q) u0 = fma(ad[q], H[(int)w.neg[q] * N + i], u0);
        double m0 = 0.0, m1 = 0.0;
        const double* Mi = MtM + i * N;
#pragma unroll
        for (int j = 0; j < N; j += 2) {
          m0 = fma(Mi[j], Fd[j], m0);
          if (j + 1 < N) m1 = fma(Mi[j + 1], Fd[j + 1], m1);
        }
        rmax = fmax(rmax, fabs(w.b[i] - ((m0 + m1) + ((u0 + u1) + (u2 + u3)))));
        bmax = fmax(bmax, fabs(w.b[i]));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
      bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
    }
    ++checked;
    if (tol <= 0.0 || rmax > tol * bmax) {  // tol 0: every voxel
      __syncwarp();
      const bool ok = solve_fp64<N>(P.sc, k, w, slot, lane);
      for (int c = lane; c < N; c += 32) P.F[v * Dims<N>::HS + c] = w.F[c];
      if (lane == 0) P.status[v] = (uint8_t)(st | CSD_STATUS_FP64 | (ok ? 0 : CSD_STATUS_CHOLFAIL));
      ++resolved;
    }
    __syncwarp();
  }
  if (lane == 0 && (checked || resolved)) {
    atomicAdd(ctr, checked);
    atomicAdd(ctr + 1, resolved);
  }
}

template <int N>
__global__ void csd_state_fod_kernel(const float* F, const uint8_t* status, const uint16_t* iters, const uint32_t* old,
                                     int nw, long long n, float* fod, long long fod_stride, uint8_t* st_out,
                                     uint8_t* it_out, uint32_t* neg_out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * N) return;
  const long long v = i / N;
  const int c = (int)(i - v * N);
  const uint8_t s0 = status[v] & 0x0F;
  const bool solved = s0 != CSD_STATUS_MASKED && s0 != CSD_STATUS_NONFINITE;  // else no F is kept
  fod[v * fod_stride + c] = solved ? F[v * Dims<N>::HS + c] : 0.f;
  if (c == 0) {
    uint8_t s = status[v];
    if ((s & 0x0F) == 0x0F) s = (uint8_t)(CSD_STATUS_NITER | (s & 0x70));  // still iterating
    else s = (uint8_t)(s & 0x7F);
    if (st_out) st_out[v] = s;
    if (it_out) it_out[v] = (uint8_t)(iters[v] > 255 ? 255 : iters[v]);
    if (neg_out)
      for (int p = 0; p < nw; ++p) neg_out[v * nw + p] = solved ? old[v * nw + p] : 0u;
  }
}

}  // namespace csdb200

// ---------------------------------------------------------------------------
// shared tables

struct csd_shared {
  HostShared h;
  uint64_t id = 0;               // unique per object: caches key on it, not on the address
  double cond_thr = 1e6;
  int refine = 3;
  int device = -1;               // device holding the tables (-1: not uploaded yet)
  std::mutex upload_mu;
  int HS = 0, WSZ = 0;
  int hexp = 0;                    // the FP16 tables hold HR_trans * 2^-hexp (largest entry in [2^14, 2^15))
  std::vector<float> H32_host;
  std::vector<__half> H16_host;    // [2][nhr+1][HS16]: hi then lo
  std::vector<__half> Hp16_host;   // [2][npd][HS16]: projection table, hi then lo
  std::vector<__half> Htc16_host;  // tcgen05 projection table (core-matrix layout), hi then lo
  std::vector<__half> Ptc16_host;  // tcgen05 assembly table: HR_trans products in packed-W order (AsmDims)
  int pexp = 0;                    // the assembly table holds the products * 2^-pexp
  int npd = 0;                     // directions padded to a multiple of 320
  std::vector<float> MtMp_host;
  std::vector<float> rconvT_host;
  std::vector<float> M32_host;
  float* H32 = nullptr;
  __half* H16 = nullptr;
  __half* Hp16 = nullptr;
  __half* Htc16 = nullptr;
  __half* Ptc16 = nullptr;
  double* H64 = nullptr;
  float* MtMp = nullptr;
  double* MtM64 = nullptr;
  float* rconvT = nullptr;
  float* M32 = nullptr;
  int* dwis = nullptr;
};

static bool supported_nsh(int n) { return n == 6 || n == 15 || n == 28 || n == 45 || n == 66 || n == 91; }

extern "C" void csd_params_init(csd_params* p) {
  if (!p) return;
  p->lmax = 0;
  p->niter = 50;
  p->neg_lambda = 1.0;
  p->norm_lambda = 1.0;
  p->threshold = 0.0;
  p->filter = nullptr;
  p->n_filter = 0;
  p->bzero_threshold = 10.0;
  p->bvalue_epsilon = 80.0;
  p->fp64_condition = 1e6;
  p->refine = 3;
  p->shells = nullptr;
  p->n_shells = 0;
}

template <typename T>
static int upload(T** dst, const std::vector<T>& src) {
  CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(dst), std::max<size_t>(src.size(), 1) * sizeof(T)));
  if (!src.empty()) CUDA_TRY(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

static std::vector<double> builtin_hr_dirs();

extern "C" int csd_shared_create(const csd_params* p, const double* grad, int n_volumes, const double* response,
                                 int n_response, const double* hr_dirs, int n_hr, csd_shared** out) {
  if (!out) return fail(CSD_ERR_INVALID, "csd_shared_create: out is NULL");
  *out = nullptr;
  csd_params def;
  csd_params_init(&def);
  if (!p) p = &def;
  SharedParams sp;
  sp.lmax = p->lmax;
  sp.niter = p->niter;
  sp.neg_lambda = p->neg_lambda;
  sp.norm_lambda = p->norm_lambda;
  sp.threshold = p->threshold;
  if (p->filter && p->n_filter > 0) sp.filter.assign(p->filter, p->filter + p->n_filter);
  sp.bzero_threshold = p->bzero_threshold;
  sp.bvalue_epsilon = p->bvalue_epsilon;
  if (p->shells && p->n_shells > 0) sp.shells.assign(p->shells, p->shells + p->n_shells);
  std::vector<double> hr;
  if (hr_dirs) {
    if (n_hr <= 0) return fail(CSD_ERR_INVALID, "n_hr must be positive");
    hr.assign(hr_dirs, hr_dirs + 2 * (size_t)n_hr);
  } else {
    hr = builtin_hr_dirs();
    n_hr = (int)(hr.size() / 2);
  }
  std::unique_ptr<csd_shared> s(new csd_shared);
  static std::atomic<uint64_t> next_id{1};
  s->id = next_id++;
  try {
    s->h = build_shared(sp, grad, n_volumes, response, n_response, hr.data(), n_hr);
  } catch (const std::exception& e) {
    return fail(CSD_ERR_INVALID, e.what());
  }
  const HostShared& h = s->h;
  if (!supported_nsh(h.nsh)) return fail(CSD_ERR_UNSUPPORTED, "lmax above the compiled maximum (12)");
  if (h.nhr > kMaxHR) return fail(CSD_ERR_UNSUPPORTED, "more than 512 constraint directions");
  if (h.ndw > kMaxDW) return fail(CSD_ERR_UNSUPPORTED, "more than 512 DW volumes in the shell");
  if (h.niter > 255 * 4) return fail(CSD_ERR_INVALID, "niter out of range [0,1000]");
  s->cond_thr = p->fp64_condition > 0 ? p->fp64_condition : 1e6;
  if (p->refine < 0 || p->refine > 3) return fail(CSD_ERR_INVALID, "refine must be 0, 1, 2 or 3");
  s->refine = p->refine;
  const int n = h.nsh;
  s->HS = hr_stride(n);
  s->WSZ = packoff(n);
  // HR_trans fp32, rows padded to HS with zeros
  s->H32_host.assign((size_t)h.nhr * s->HS, 0.f);
  for (int d = 0; d < h.nhr; ++d)
    for (int c = 0; c < n; ++c) s->H32_host[(size_t)d * s->HS + c] = (float)h.HR[(size_t)d * n + c];
  // FP16 hi/lo split of HR_trans for the tensor-core assembly, plus a zero
  // row.  HR_trans grows with the response (csd.h:175-180: the constraint
  // multiplier is 50 r0 / 300), so the split is taken of HR_trans * 2^-hexp,
  // an exact power of two that puts the largest entry in [2^14, 2^15): the
  // hi halves stay below FP16's 65504 and the lo halves of the entries that
  // matter stay normal at any response scale.  The kernels scale back exactly.
  double hmax = 0.0;
  for (double x : h.HR) hmax = std::max(hmax, std::fabs(x));
  if (!(hmax > 0.0) || !std::isfinite(hmax)) return fail(CSD_ERR_INVALID, "constraint matrix is zero or not finite");
  s->hexp = std::ilogb(hmax) - 14;
  if (s->hexp < -60 || s->hexp > 60) return fail(CSD_ERR_UNSUPPORTED, "response scale out of the supported range");
  const double hdown = std::ldexp(1.0, -s->hexp);
  const int HS16 = hr_stride16(n);
  s->H16_host.assign((size_t)2 * (h.nhr + 1) * HS16, __float2half_rn(0.f));
  for (int d = 0; d < h.nhr; ++d)
    for (int c = 0; c < n; ++c) {
      const double x = h.HR[(size_t)d * n + c] * hdown;
      const __half hi = __float2half_rn((float)x);
      const __half lo = __float2half_rn((float)(x - (double)__half2float(hi)));
      s->H16_host[(size_t)d * HS16 + c] = hi;
      s->H16_host[(size_t)(h.nhr + 1 + d) * HS16 + c] = lo;
    }
  s->npd = (h.nhr + 319) / 320 * 320;
  s->Hp16_host.assign((size_t)2 * s->npd * HS16, __float2half_rn(0.f));
  for (int d = 0; d < h.nhr; ++d)
    for (int c = 0; c < n; ++c) {
      s->Hp16_host[(size_t)d * HS16 + c] = s->H16_host[(size_t)d * HS16 + c];
      s->Hp16_host[(size_t)(s->npd + d) * HS16 + c] = s->H16_host[(size_t)(h.nhr + 1 + d) * HS16 + c];
    }
  if (h.nhr <= 320) {
    // canonical K-major core matrices: [K chunk][row group of 8][row][8 halves]
    const int KC = 2 * ((n + 15) / 16);
    const size_t per = (size_t)KC * 320 * 8;
    s->Htc16_host.assign(2 * per, __float2half_rn(0.f));
    for (int kc = 0; kc < KC; ++kc)
      for (int d = 0; d < h.nhr; ++d)
        for (int e = 0; e < 8; ++e) {
          const int c = 8 * kc + e;
          if (c >= n) continue;
          const size_t o = ((size_t)(kc * 40 + d / 8) * 8 + (d % 8)) * 8 + e;
          s->Htc16_host[o] = s->H16_host[(size_t)d * HS16 + c];
          s->Htc16_host[per + o] = s->H16_host[(size_t)(h.nhr + 1 + d) * HS16 + c];
        }
  }
  if (h.nhr <= kAsmK) {
    // rank-k assembly as one dense product per tile (csd_assemble_tc_kernel):
    // column c = packoff(i) + j (j <= i) of W gets sum_d mask_d * h_d[i] h_d[j],
    // so the table holds the products h_d[i] h_d[j] (FP64, scaled by an exact
    // power of two that puts the largest in [2^14, 2^15)) split into FP16
    // hi + lo, padding columns zero, laid out as the kernel's shared-memory
    // stages: [chunk][slab][hi | lo][K chunk of 8][column][8 halves]
    s->pexp = std::ilogb(hmax * hmax) - 14;
    const double pdown = std::ldexp(1.0, -s->pexp);
    const AsmShape a = asm_shape(n);
    const size_t half_stage = (size_t)(kAsmSlabK / 8) * a.nc * 8;  // halves of one of hi / lo
    s->Ptc16_host.assign((size_t)a.nch * kAsmSlabs * 2 * half_stage, __float2half_rn(0.f));
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) {
        const int c = packoff(i) + j, ch = c / a.nc, cl = c % a.nc;
        for (int d = 0; d < h.nhr; ++d) {
          const double x = h.HR[(size_t)d * n + i] * h.HR[(size_t)d * n + j] * pdown;
          const __half hi = __float2half_rn((float)x);
          const __half lo = __float2half_rn((float)(x - (double)__half2float(hi)));
          const int sl = d / kAsmSlabK, kc = (d % kAsmSlabK) / 8, e = d % 8;
          const size_t o = ((size_t)(ch * kAsmSlabs + sl) * 2) * half_stage + ((size_t)kc * a.nc + cl) * 8 + e;
          s->Ptc16_host[o] = hi;
          s->Ptc16_host[o + half_stage] = lo;
        }
      }
  }
  s->MtMp_host.assign((size_t)s->WSZ, 0.f);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) s->MtMp_host[packoff(i) + j] = (float)h.MtM[(size_t)i * n + j];
  s->rconvT_host.assign((size_t)h.ndw * h.ninit, 0.f);
  for (int r = 0; r < h.ninit; ++r)
    for (int t = 0; t < h.ndw; ++t) s->rconvT_host[(size_t)t * h.ninit + r] = (float)h.rconv[(size_t)r * h.ndw + t];
  s->M32_host.assign(h.M.size(), 0.f);
  for (size_t i = 0; i < h.M.size(); ++i) s->M32_host[i] = (float)h.M[i];
  *out = s.release();
  return CSD_OK;
}

// The tables go to the device on first use (so the host precompute can be
// created and inspected without a GPU); later calls must use the same device.
static int ensure_device(const csd_shared* cs) {
  csd_shared* s = const_cast<csd_shared*>(cs);
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(s->upload_mu);
  if (s->device == dev) return 0;
  if (s->device >= 0) return fail(CSD_ERR_INVALID, "shared tables live on another device");
  int rc;
  const HostShared& h = s->h;
  if ((rc = upload(&s->H32, s->H32_host))) return rc;
  if ((rc = upload(&s->H16, s->H16_host))) return rc;
  if ((rc = upload(&s->Hp16, s->Hp16_host))) return rc;
  if (!s->Htc16_host.empty() && (rc = upload(&s->Htc16, s->Htc16_host))) return rc;
  if (!s->Ptc16_host.empty() && (rc = upload(&s->Ptc16, s->Ptc16_host))) return rc;
  if ((rc = upload(&s->H64, h.HR))) return rc;
  if ((rc = upload(&s->MtMp, s->MtMp_host))) return rc;
  if ((rc = upload(&s->MtM64, h.MtM))) return rc;
  if ((rc = upload(&s->rconvT, s->rconvT_host))) return rc;
  if ((rc = upload(&s->M32, s->M32_host))) return rc;
  if ((rc = upload(&s->dwis, h.dwis))) return rc;
  s->device = dev;
  return 0;
}

extern "C" void csd_shared_destroy(csd_shared* s) {
  if (!s) return;
  if (s->device >= 0) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(s->device);
    cudaFree(s->H32);
    cudaFree(s->H16);
    cudaFree(s->Hp16);
    cudaFree(s->Htc16);
    cudaFree(s->Ptc16);
    cudaFree(s->H64);
    cudaFree(s->MtMp);
    cudaFree(s->MtM64);
    cudaFree(s->rconvT);
    cudaFree(s->M32);
    cudaFree(s->dwis);
    cudaSetDevice(cur);
  }
  delete s;
}

extern "C" int csd_shared_nsh(const csd_shared* s) { return s ? s->h.nsh : fail(CSD_ERR_INVALID, "NULL shared"); }

extern "C" int csd_shared_info(const csd_shared* s, int* info) {
  if (!s || !info) return fail(CSD_ERR_INVALID, "NULL argument");
  const HostShared& h = s->h;
  const int v[8] = {h.lmax, h.lmax_response, h.lmax_data, h.nsh, h.ninit, h.ndw, h.nhr, h.niter};
  std::memcpy(info, v, sizeof(v));
  return CSD_OK;
}

extern "C" int csd_shared_dwis(const csd_shared* s, int* out) {
  if (!s || !out) return fail(CSD_ERR_INVALID, "NULL argument");
  std::copy(s->h.dwis.begin(), s->h.dwis.end(), out);
  return CSD_OK;
}

extern "C" int csd_shared_matrix(const csd_shared* s, int which, double* out) {
  if (!s || !out) return fail(CSD_ERR_INVALID, "NULL argument");
  const HostShared& h = s->h;
  switch (which) {
    case 0: std::copy(h.rconv.begin(), h.rconv.end(), out); break;
    case 1: std::copy(h.M.begin(), h.M.end(), out); break;
    case 2: std::copy(h.MtM.begin(), h.MtM.end(), out); break;
    case 3: std::copy(h.HR.begin(), h.HR.end(), out); break;
    case 4: out[0] = h.threshold; out[1] = h.norm_lambda; out[2] = h.neg_lambda; break;
    default: return fail(CSD_ERR_INVALID, "unknown matrix id");
  }
  return CSD_OK;
}

// ---------------------------------------------------------------------------
// per-(device, stream) workspace: work counter and FP64 fallback slots

namespace {
struct Workspace {
  unsigned long long* queue = nullptr;   // kMaxQueues counters
  double* fp64 = nullptr;
  size_t fp64_doubles = 0;
  // device staging for the host-buffer entry point
  float* d_dwi = nullptr;
  size_t d_dwi_n = 0;
  float* d_fod = nullptr;
  size_t d_fod_n = 0;
  uint8_t* d_small = nullptr;
  size_t d_small_n = 0;
  cudaStream_t streams[2] = {nullptr, nullptr};
};
std::mutex g_ws_mu;
std::map<std::pair<int, void*>, Workspace> g_ws;

int get_ws(void* stream, Workspace** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_ws_mu);
  Workspace& w = g_ws[{dev, stream}];
  if (!w.queue) CUDA_TRY(cudaMalloc(&w.queue, 64 * sizeof(unsigned long long)));
  *out = &w;
  return 0;
}

template <typename T>
int grow(T** p, size_t* have, size_t need) {
  if (*have >= need) return 0;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *have = 0;
  if (cudaMalloc(reinterpret_cast<void**>(p), need * sizeof(T)) != cudaSuccess)
    return fail(CSD_ERR_NOMEM, "device allocation failed");
  *have = need;
  return 0;
}

struct LaunchShape {
  int warps = 0, blocks = 0;
  size_t smem = 0;
};

template <int N>
int launch_persistent(const SolveParams& P, size_t smem, int warps, int blocks, cudaStream_t st) {
  CUDA_TRY(cudaFuncSetAttribute(csd_persistent_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem));
  csd_persistent_kernel<N><<<blocks, warps * 32, smem, st>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

template <int N>
int shape_for(int nhr, long long total, LaunchShape* ls) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  int smem_max = 0, nsm = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t hbytes = (size_t)htab_bytes<N>(nhr);
  const size_t wb = warp_ws_bytes<N>();
  if (hbytes + wb > (size_t)smem_max) return fail(CSD_ERR_UNSUPPORTED, "constraint set too large for shared memory");
  int warps = (int)std::min<size_t>(Dims<N>::THREADS / 32, ((size_t)smem_max - hbytes) / wb);
  if (g_tune_persistent_warps > 0) warps = std::min(warps, g_tune_persistent_warps);
  ls->warps = warps;
  ls->smem = hbytes + wb * warps;
  long long need_blocks = (total + warps - 1) / warps;
  ls->blocks = (int)std::max<long long>(1, std::min<long long>(nsm, need_blocks));
  return 0;
}

int dispatch(int nsh, const SolveParams& P, cudaStream_t st, Workspace* ws) {
  LaunchShape ls;
  int rc = 0;
  size_t wsz = 0;
  switch (nsh) {
#define CSD_CASE(NN)                                                    \
  case NN:                                                              \
    if ((rc = shape_for<NN>(P.nhr, P.total, &ls))) return rc;          \
    wsz = Dims<NN>::WSZ;                                                \
    break;
    CSD_CASE(6) CSD_CASE(15) CSD_CASE(28) CSD_CASE(45) CSD_CASE(66) CSD_CASE(91)
#undef CSD_CASE
    default:
      return fail(CSD_ERR_UNSUPPORTED, "unsupported nSH");
  }
  if ((rc = grow(&ws->fp64, &ws->fp64_doubles, (size_t)ls.blocks * ls.warps * wsz))) return rc;
  SolveParams Q = P;
  Q.fp64_scratch = ws->fp64;
  switch (nsh) {
#define CSD_CASE(NN) \
  case NN: return launch_persistent<NN>(Q, ls.smem, ls.warps, ls.blocks, st);
    CSD_CASE(6) CSD_CASE(15) CSD_CASE(28) CSD_CASE(45) CSD_CASE(66) CSD_CASE(91)
#undef CSD_CASE
  }
  return 0;
}

}  // namespace

static Scheme scheme_of(const csd_shared* s) {
  Scheme sc;
  sc.H32 = s->H32;
  sc.H16 = s->H16;
  sc.H64 = s->H64;
  sc.MtMp = s->MtMp;
  sc.MtM64 = s->MtM64;
  sc.rconvT = s->rconvT;
  sc.M32 = s->M32;
  sc.dwis = s->dwis;
  sc.ndw = s->h.ndw;
  sc.ninit = s->h.ninit;
  sc.niter = s->h.niter;
  sc.threshold = (float)s->h.threshold;
  sc.hscale = pow2f(s->hexp);
  return sc;
}

static int g_refine = -1;  // test override of csd_params::refine (-1 = none)
static int refine_of(const csd_shared* s) { return g_refine >= 0 ? g_refine : s->refine; }

extern "C" int csd_solve(const csd_shared* const* shared, const csd_volume* volumes, int n_volumes, void* stream) {
  if (n_volumes < 0 || (n_volumes > 0 && (!shared || !volumes)))
    return fail(CSD_ERR_INVALID, "csd_solve: invalid volume list");
  if (n_volumes == 0) return CSD_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int nsh = shared[0] ? shared[0]->h.nsh : 0;
  const int nhr = shared[0] ? shared[0]->h.nhr : 0;
  for (int i = 0; i < n_volumes; ++i) {
    const csd_shared* s = shared[i];
    const csd_volume& v = volumes[i];
    if (!s) return fail(CSD_ERR_INVALID, "csd_solve: NULL shared");
    if (s->h.nsh != nsh || s->h.nhr != nhr)
      return fail(CSD_ERR_INVALID, "csd_solve: all volumes of one call must share nSH and the constraint set size");
    if (v.n_voxels < 0) return fail(CSD_ERR_INVALID, "csd_solve: negative voxel count");
    if (v.n_voxels > 0 && (!v.dwi || !v.fod)) return fail(CSD_ERR_INVALID, "csd_solve: NULL dwi or fod");
    if (v.fod_stride < nsh) return fail(CSD_ERR_INVALID, "csd_solve: fod_stride smaller than nSH");
    if (v.voxel_stride < 0 || v.volume_stride < 0) return fail(CSD_ERR_INVALID, "csd_solve: negative stride");
  }
  Workspace* ws = nullptr;
  int rc = get_ws(stream, &ws);
  if (rc) return rc;
  for (int i = 0; i < n_volumes; ++i)
    if ((rc = ensure_device(shared[i]))) return rc;
  // group volumes by identical constraint tables; each group is one launch
  std::vector<int> order(n_volumes);
  std::vector<char> done(n_volumes, 0);
  for (int i = 0; i < n_volumes; ++i) {
    if (done[i]) continue;
    std::vector<int> group;
    for (int j = i; j < n_volumes; ++j)
      if (!done[j] && (shared[j] == shared[i] || shared[j]->H32_host == shared[i]->H32_host)) {
        group.push_back(j);
        done[j] = 1;
      }
    for (size_t g0 = 0; g0 < group.size(); g0 += kMaxVolumesPerLaunch) {
      const size_t g1 = std::min(group.size(), g0 + kMaxVolumesPerLaunch);
      SolveParams P;
      std::memset(&P, 0, sizeof(P));
      P.nhr = nhr;
      P.nw = (nhr + 31) / 32;
      P.refine = refine_of(shared[group[g0]]);
      P.fast_cycles = g_fast_cycles == 1;
      P.cond_thr = (float)shared[group[g0]]->cond_thr;
      long long total = 0;
      int nv = 0;
      for (size_t q = g0; q < g1; ++q) {
        const int j = group[q];
        const csd_volume& v = volumes[j];
        if (v.n_voxels == 0) continue;
        VolumeDesc& d = P.vol[nv++];
        d.sc = scheme_of(shared[j]);
        d.dwi = v.dwi;
        d.n_voxels = v.n_voxels;
        d.vox_stride = v.voxel_stride;
        d.vol_stride = v.volume_stride;
        d.first = total;
        d.mask = v.mask;
        d.warm = v.warm_negmask;
        d.fod = v.fod;
        d.fod_stride = v.fod_stride;
        d.status = v.status;
        d.iters = v.iterations;
        d.negmask = v.negmask;
        total += v.n_voxels;
      }
      if (nv == 0) continue;
      P.n_vol = nv;
      P.total = total;
      P.queue = ws->queue;
      CUDA_TRY(cudaMemsetAsync(ws->queue, 0, sizeof(unsigned long long), st));
      if ((rc = dispatch(nsh, P, st, ws))) return rc;
    }
  }
  return CSD_OK;
}

// ---------------------------------------------------------------------------
// host-buffer entry point: slabs of voxels staged host -> device -> host with
// copies on two streams overlapping the solve of the neighbouring slab.

extern "C" int csd_dwi2fod_host(const csd_shared* s, const float* dwi, int64_t n_voxels, const uint8_t* mask,
                                float* fod, uint8_t* status, uint8_t* iterations) {
  if (!s || n_voxels < 0 || (n_voxels > 0 && (!dwi || !fod)))
    return fail(CSD_ERR_INVALID, "csd_dwi2fod_host: invalid argument");
  if (n_voxels == 0) return CSD_OK;
  const int nvol = s->h.nvol, nsh = s->h.nsh;
  Workspace* ws = nullptr;
  int rc = get_ws(reinterpret_cast<void*>(1), &ws);  // private key for this entry point
  if (rc) return rc;
  if (!ws->streams[0]) {
    CUDA_TRY(cudaStreamCreateWithFlags(&ws->streams[0], cudaStreamNonBlocking));
    CUDA_TRY(cudaStreamCreateWithFlags(&ws->streams[1], cudaStreamNonBlocking));
  }
  cudaStream_t* streams = ws->streams;
  if ((rc = grow(&ws->d_dwi, &ws->d_dwi_n, (size_t)n_voxels * nvol))) return rc;
  if ((rc = grow(&ws->d_fod, &ws->d_fod_n, (size_t)n_voxels * nsh))) return rc;
  if ((rc = grow(&ws->d_small, &ws->d_small_n, (size_t)n_voxels * 3))) return rc;
  uint8_t* d_mask = ws->d_small;
  uint8_t* d_status = ws->d_small + n_voxels;
  uint8_t* d_iters = ws->d_small + 2 * n_voxels;
  const int64_t nslab = std::min<int64_t>(8, std::max<int64_t>(1, n_voxels / 65536));
  const int64_t per = (n_voxels + nslab - 1) / nslab;
  const csd_shared* sh[1] = {s};
  for (int64_t k = 0; k < nslab; ++k) {
    const int64_t a = k * per, n = std::min(per, n_voxels - a);
    if (n <= 0) break;
    cudaStream_t st = streams[k & 1];
    CUDA_TRY(cudaMemcpyAsync(ws->d_dwi + a * nvol, dwi + a * nvol, (size_t)n * nvol * sizeof(float),
                             cudaMemcpyHostToDevice, st));
    if (mask) CUDA_TRY(cudaMemcpyAsync(d_mask + a, mask + a, (size_t)n, cudaMemcpyHostToDevice, st));
    csd_volume v;
    std::memset(&v, 0, sizeof(v));
    v.dwi = ws->d_dwi + a * nvol;
    v.n_voxels = n;
    v.voxel_stride = nvol;
    v.volume_stride = 1;
    v.mask = mask ? d_mask + a : nullptr;
    v.fod = ws->d_fod + a * nsh;
    v.fod_stride = nsh;
    v.status = status ? d_status + a : nullptr;
    v.iterations = iterations ? d_iters + a : nullptr;
    if ((rc = csd_solve(sh, &v, 1, st))) return rc;
    CUDA_TRY(cudaMemcpyAsync(fod + a * nsh, ws->d_fod + a * nsh, (size_t)n * nsh * sizeof(float),
                             cudaMemcpyDeviceToHost, st));
    if (status) CUDA_TRY(cudaMemcpyAsync(status + a, d_status + a, (size_t)n, cudaMemcpyDeviceToHost, st));
    if (iterations) CUDA_TRY(cudaMemcpyAsync(iterations + a, d_iters + a, (size_t)n, cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(cudaStreamSynchronize(streams[0]));
  CUDA_TRY(cudaStreamSynchronize(streams[1]));
  return CSD_OK;
}

// Launch-shape knobs (set by the autotuner): which = 0 persistent-kernel
// warps per block, 1 phased solve-kernel warps per block, 2 projection
// blocks per SM; value 0 restores the default.  Results do not depend on
// them (each voxel's arithmetic is the same whatever warp runs it).
extern "C" int csd_set_launch_config(int which, int value) {
  if (value < 0 || value > 64) return fail(CSD_ERR_INVALID, "csd_set_launch_config: value out of range");
  switch (which) {
    case 0: g_tune_persistent_warps = value; break;
    case 1: g_tune_solve_warps = value; break;
    case 2: g_tune_proj_blocks_per_sm = value; break;
    case 3:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: projection kind is 0, 1 or 2");
      g_proj_kind = value;
      break;
    case 4:
      if (value > 3) return fail(CSD_ERR_INVALID, "csd_set_launch_config: solve kind is 0, 1, 2 or 3");
      g_solve_kind = value;
      break;
    case 5:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: set kind is 0, 1 or 2");
      g_set_kind = value;
      break;
    case 6:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: inference kind is 0, 1 or 2");
      csdb200::g_mlp_infer_kind = value;
      break;
    case 7:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: cycle jumping is 0 (default), 1 on or 2 off");
      g_fast_cycles = value;
      break;
    case 8:
      if (value > 16) return fail(CSD_ERR_INVALID, "csd_set_launch_config: at most 16 slabs");
      g_host_slabs = value;
      break;
    case 9:
      if (value > 3) return fail(CSD_ERR_INVALID, "csd_set_launch_config: amp2sh kernel is 0, 1, 2 or 3");
      csdb200::g_amp2sh_kind = value;
      break;
    case 10:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: factor reuse is 0 (default), 1 on or 2 off");
      g_reuse = value;
      break;
    case 11:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: asynchronous host slabs are 0 (default), 1 on or 2 off");
      g_host_async = value;
      break;
    case 12:
      if (value > 2) return fail(CSD_ERR_INVALID, "csd_set_launch_config: assembly is 0 (default), 1 mma.sync or 2 tcgen05");
      g_asm_kind = value;
      break;
    case 13:
      if (value > 16) return fail(CSD_ERR_INVALID, "csd_set_launch_config: at most 16 slabs computing at once");
      g_host_conc = value;
      break;
    default: return fail(CSD_ERR_INVALID, "csd_set_launch_config: unknown knob");
  }
  return CSD_OK;
}

// Profiling hook: per-phase cycle totals of the persistent kernel since the
// last reset (only in a build with -DCSD_PHASE_TIMERS; returns -5 otherwise).
extern "C" int csd_debug_phase_cycles(unsigned long long* out, int reset) {
#ifdef CSD_PHASE_TIMERS
  CUDA_TRY(cudaMemcpyFromSymbol(out, g_phase_cycles, sizeof(unsigned long long) * 16));
  if (reset) {
    unsigned long long z[16] = {};
    CUDA_TRY(cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z)));
  }
  return CSD_OK;
#else
  (void)out;
  (void)reset;
  return fail(CSD_ERR_UNSUPPORTED, "built without CSD_PHASE_TIMERS");
#endif
}

// test hook: refinement mode
extern "C" int csd_debug_set_refine(int mode) {
  g_refine = mode < 0 ? -1 : (mode > 3 ? 3 : mode);
  return CSD_OK;
}


// ---------------------------------------------------------------------------
// csd_state_*: per-step surface (CSD::set / iterate / FOD over a batch)

// passes enqueued by csd_state_run between two reads of the active count
static constexpr int kRunBatch = 16;

struct csd_state {
  const csd_shared* sh = nullptr;
  int64_t cap = 0, n = 0, n_active = 0;
  int use_warm = 0;
  float* F = nullptr;
  double* b = nullptr;
  uint32_t* old = nullptr;
  uint32_t* old2 = nullptr;
  uint32_t* newm = nullptr;
  uint32_t* warm = nullptr;
  uint8_t* status = nullptr;
  uint16_t* iters = nullptr;
  uint16_t* cyc = nullptr;
  float* Lst = nullptr;       // first-solve factors of warm-started voxels (allocated on first warm use)
  uint8_t* fac = nullptr;     // 1 = Lst holds the voxel's warm-set factor
  size_t lst_floats = 0;      // ReuseLayout<nSH>::LSZ
  int reuse_warps = 0;        // launch shape of csd_solve_reuse_kernel
  size_t reuse_smem = 0;
  int* act[2] = {nullptr, nullptr};
  int* slist = nullptr;
  int* rlist = nullptr;       // the solve list's voxels the reuse kernel leaves to the full kernel
  int* rcount = nullptr;      // device: their count, per pass of a csd_state_run batch
  int* counter = nullptr;
  int cur = 0;
  double* fp64 = nullptr;
  int blocks = 0, warps = 0;
  size_t smem = 0;
  int gwarps[2] = {0, 0};     // grouped solve kernel, 16 / 8 lanes per voxel (0: unavailable)
  size_t set_smem = 0;        // tiled set kernel's shared memory (0: tables too large for it)
  size_t gsmem[2] = {0, 0};
  int proj_blocks = 0;
  size_t proj_smem = 0;
  float* Wg = nullptr;        // systems assembled by csd_assemble_tc_kernel, wg_entries rows of packoff(nSH)
  long long wg_entries = 0;
  int pre_warps = 0;          // launch shape of csd_solve_kernel<N, true>
  size_t pre_smem = 0;
  static constexpr int kAsmEv = 64;   // timed assembly launches between two host synchronisations
  cudaEvent_t aev[2 * kAsmEv] = {};
  int n_aev = 0;
  bool time_asm = false;      // record events around csd_assemble_tc_kernel (synchronous runs only)
  double ms_asm = 0;          // device time of csd_assemble_tc_kernel since the last set()
  long long asm_launches = 0;
  long long passes = 0, projected = 0, solved = 0;  // work counters since the last set()
  unsigned long long* stats = nullptr;              // device: sum |neg|, solves
  unsigned long long* chk = nullptr;                // device: voxels checked, re-solved (csd_state_check)
  long long fp64_slots = 0;                         // warps' FP64 slots in fp64
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int* pcount = nullptr;                            // device: per-pass counts of csd_state_run
  int* acount = nullptr;                            // device: per-pass counts of csd_state_run_async
  int* arcount = nullptr;                           //   and its rest-list counts
  int async_passes = 0;                             // passes acount has room for
  int async_cur = 0;                                // list the last async run ended on
  cudaEvent_t bev[3 * kRunBatch + 1] = {};          // kernel boundaries of one csd_state_run batch
  double ms_set = 0, ms_project = 0, ms_solve = 0;  // device time of the kernels since the last set()
  double ms_reuse = 0;                              // of which in csd_solve_reuse_kernel
  long long launches = 0;
};

namespace {
template <int N>
int state_shape(csd_state* st) {
  LaunchShape ls;
  {
    int dev = 0, smem_max = 0, nsm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const size_t hbytes = (size_t)htab_bytes<N>(st->sh->h.nhr, false);
    const size_t wb = warp_ws_bytes<N>();
    if (hbytes + wb > (size_t)smem_max) return fail(CSD_ERR_UNSUPPORTED, "constraint set too large for shared memory");
    ls.warps = (int)std::min<size_t>(Dims<N>::SOLVE_THREADS / 32, ((size_t)smem_max - hbytes) / wb);
    ls.smem = hbytes + wb * ls.warps;
    ls.blocks = nsm;
  }
  st->blocks = ls.blocks;
  st->warps = ls.warps;
  st->smem = ls.smem;
  int maxw = ls.warps;
  if constexpr (N <= 45) {
    int dev = 0, smem_max = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t hbytes = (size_t)htab_bytes<N>(st->sh->h.nhr, false);
    const size_t wb[2] = {(size_t)GroupWSLayout<N, 2>::WARP, (size_t)GroupWSLayout<N, 4>::WARP};
    const int cap[2] = {GroupSolveThreads<16>::value / 32, GroupSolveThreads<8>::value / 32};
    for (int i = 0; i < 2; ++i) {
      if (hbytes + wb[i] > (size_t)smem_max) continue;
      st->gwarps[i] = (int)std::min<size_t>(cap[i], ((size_t)smem_max - hbytes) / wb[i]);
      st->gsmem[i] = hbytes + wb[i] * st->gwarps[i];
      maxw = std::max(maxw, st->gwarps[i]);
    }
    if (st->gwarps[0])
      CUDA_TRY(cudaFuncSetAttribute(csd_solve_group_kernel<N, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)st->gsmem[0]));
    if (st->gwarps[1])
      CUDA_TRY(cudaFuncSetAttribute(csd_solve_group_kernel<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)st->gsmem[1]));
  }
  if (st->sh->Ptc16) {
    // tcgen05 assembly ahead of a table-free solve kernel: the solve list in
    // chunks of wg_entries systems (at most ~4 GB of them)
    int dev = 0, smem_max = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t wb = warp_ws_bytes<N>();
    const size_t asm_smem = std::max<size_t>(asm_smem_bytes(N), 120 * 1024);  // one block (one TMEM owner) an SM
    if (asm_smem <= (size_t)smem_max && wb <= (size_t)smem_max) {
      st->pre_warps = (int)std::min<size_t>(PreSolveThreads<N>::value / 32, (size_t)smem_max / wb);
      st->pre_smem = wb * st->pre_warps;
      maxw = std::max(maxw, st->pre_warps);
      const long long per = (long long)Dims<N>::WSZ * (long long)sizeof(float);
      long long ent = std::min<long long>((st->cap + 127) / 128 * 128, std::max<long long>(4096, 4000000000LL / per));
      if (const char* env = std::getenv("CSD_ASM_CHUNK")) {  // smaller chunks, to exercise chunking in tests
        const long long c = std::atoll(env);
        if (c >= 128) ent = std::min(ent, c);
      }
      ent = std::max<long long>(128, ent / 128 * 128);
      CUDA_TRY(cudaMalloc(&st->Wg, (size_t)ent * per));
      st->wg_entries = ent;
      CUDA_TRY(cudaFuncSetAttribute(csd_solve_kernel<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)st->pre_smem));
      CUDA_TRY(cudaFuncSetAttribute(csd_assemble_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)asm_smem));
    }
  }
  CUDA_TRY(cudaMalloc(&st->fp64, (size_t)ls.blocks * maxw * Dims<N>::WSZ * sizeof(double)));
  st->fp64_slots = (long long)ls.blocks * maxw;
  CUDA_TRY(cudaFuncSetAttribute(csd_solve_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ls.smem));
  int dev = 0, smem_max = 0, nsm = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t psm = (size_t)2 * st->sh->npd * Dims<N>::HS16 * 2 + (size_t)2 * kProjRows * Dims<N>::HS16 * 2 +
                     (size_t)kProjRows * kMaxWords * 4 + (size_t)2 * kProjRows * 4;
  if (psm > (size_t)smem_max) return fail(CSD_ERR_UNSUPPORTED, "projection tables too large for shared memory");
  st->proj_smem = psm;
  st->proj_blocks = nsm * std::max(1, (int)(smem_max / psm));
  CUDA_TRY(cudaFuncSetAttribute(csd_project_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
  CUDA_TRY(cudaFuncSetAttribute(csd_state_set_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(8 * warp_ws_bytes<N>())));
  {
    const size_t ss = set_tile_smem(st->sh->h.ndw, st->sh->h.ninit, N);
    if (ss <= (size_t)std::min(smem_max, 200 * 1024)) {
      st->set_smem = ss;
      CUDA_TRY(cudaFuncSetAttribute(csd_state_set_tile_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
    }
  }
  {
    using RL = ReuseLayout<N>;
    const size_t per = (size_t)RL::WARP_FLOATS * sizeof(float);
    st->lst_floats = RL::LSZ;
    st->reuse_warps = (int)std::min<size_t>(RL::THREADS / 32, (size_t)smem_max / per);
    st->reuse_smem = per * st->reuse_warps;
    if (st->reuse_warps > 0)
      CUDA_TRY(cudaFuncSetAttribute(csd_solve_reuse_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)st->reuse_smem));
  }
  return 0;
}

// Device time of the csd_assemble_tc_kernel launches recorded since the last
// host synchronisation (the stream has been synchronised).
cudaError_t harvest_asm_time(csd_state* st) {
  for (int i = 0; i < st->n_aev; ++i) {
    float ms = 0.f;
    const cudaError_t e = cudaEventElapsedTime(&ms, st->aev[2 * i], st->aev[2 * i + 1]);
    if (e != cudaSuccess) return e;
    st->ms_asm += ms;
  }
  st->n_aev = 0;
  return cudaSuccess;
}

StateParams state_params(const csd_state* st) {
  StateParams P;
  std::memset(&P, 0, sizeof(P));
  P.sc = scheme_of(st->sh);
  P.nhr = st->sh->h.nhr;
  P.nw = (P.nhr + 31) / 32;
  P.npd = st->sh->npd;
  P.Hp16 = st->sh->Hp16;
  P.Htc16 = st->sh->Htc16;
  P.thr = (float)st->sh->h.threshold;
  P.hexp = st->sh->hexp;
  P.cond_thr = (float)st->sh->cond_thr;
  P.F = st->F;
  P.b = st->b;
  P.old = st->old;
  P.old2 = st->old2;
  P.newm = st->newm;
  P.warm = st->warm;
  P.use_warm = st->use_warm;
  P.status = st->status;
  P.iters = st->iters;
  P.cyc = st->cyc;
  const bool reuse = g_reuse != 2 && st->use_warm && st->Lst;
  P.Lst = reuse ? st->Lst : nullptr;
  P.fac = reuse ? st->fac : nullptr;
  P.fast_cycles = g_fast_cycles != 2;
  P.n_out = st->counter;
  P.err = st->counter + 1;
  P.stats = st->stats;
  P.fp64_scratch = st->fp64;
  P.ch = 0x7fffffff;
  return P;
}

template <int N>
int state_set_launch(csd_state* st, const StateParams& P, cudaStream_t s) {
  const int kind = g_set_kind ? g_set_kind : kSetDefault;
  if (kind == 2 && st->set_smem > 0) {
    int dev = 0, nsm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long tiles = (P.n_in + kSetTile - 1) / kSetTile;
    const int per_sm = std::max(1, (int)((228 * 1024) / (st->set_smem + 1024)));
    const int blocks = (int)std::max<long long>(1, std::min<long long>(tiles, (long long)nsm * std::min(per_sm, 8)));
    csd_state_set_tile_kernel<N><<<blocks, 256, st->set_smem, s>>>(P);
    CUDA_TRY(cudaGetLastError());
    return 0;
  }
  const int blocks = (int)std::min<long long>(4096, (P.n_in + 7) / 8);
  csd_state_set_kernel<N><<<std::max(blocks, 1), 256, 8 * warp_ws_bytes<N>(), s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_project_tc_launch(csd_state* st, const StateParams& P, cudaStream_t s) {
  constexpr int KC = 2 * Dims<N>::NRB;
  const size_t need = (size_t)2 * KC * (kTcDirs / 8) * 128 + (size_t)2 * KC * (kTcRows / 8) * 128 + 16;
  const size_t smem = std::max<size_t>(need, 120 * 1024);  // > half an SM: one block (and one TMEM owner) per SM
  CUDA_TRY(cudaFuncSetAttribute(csd_project_tc_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, nsm = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = (P.n_in + kTcRows - 1) / kTcRows;
  csd_project_tc_kernel<N><<<std::max(1, std::min(tiles, nsm)), 128, smem, s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
// The first pass's "projection" of a warm-started run: csd_warm_first_pass_kernel.
int state_warm_first_launch(const StateParams& P, cudaStream_t s) {
  int dev = 0, nsm = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const long long blocks = std::max<long long>(1, std::min<long long>((P.n_in + 255) / 256, (long long)nsm * 8));
  csd_warm_first_pass_kernel<<<(unsigned)blocks, 256, 0, s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_project_launch(csd_state* st, const StateParams& P, cudaStream_t s) {
  if ((g_proj_kind ? g_proj_kind : kProjDefault) == 2 && P.Htc16) return state_project_tc_launch<N>(st, P, s);
  const int tiles = (P.n_in + kProjRows - 1) / kProjRows;
  int pb = st->proj_blocks;
  if (g_tune_proj_blocks_per_sm > 0) {
    int dev = 0, nsm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    pb = std::min(pb, nsm * g_tune_proj_blocks_per_sm);
  }
  csd_project_kernel<N><<<std::max(1, std::min(tiles, pb)), 256, st->proj_smem, s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_solve_launch(csd_state* st, const StateParams& P, cudaStream_t s) {
  const int kind = g_solve_kind ? g_solve_kind : kSolveDefault;
  if constexpr (N <= 45) {
    const int gi = kind == 2 ? 0 : kind == 3 ? 1 : -1;
    if (gi >= 0 && st->gwarps[gi] > 0) {
      const int vpw = gi == 0 ? 2 : 4;  // voxels per warp
      const int gw = st->gwarps[gi];
      const int need = (int)std::min<long long>(st->blocks, (P.n_in + (long long)gw * vpw - 1) / ((long long)gw * vpw));
      if (gi == 0)
        csd_solve_group_kernel<N, 16><<<std::max(need, 1), gw * 32, st->gsmem[0], s>>>(P);
      else
        csd_solve_group_kernel<N, 8><<<std::max(need, 1), gw * 32, st->gsmem[1], s>>>(P);
      CUDA_TRY(cudaGetLastError());
      return 0;
    }
  }
  if ((g_asm_kind ? g_asm_kind : kAsmDefault) == 2 && st->Wg && P.n_in > 0) {
    // systems of each chunk of the list assembled on tcgen05, then solved
    int dev = 0, nsm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const size_t asm_smem = std::max<size_t>(asm_smem_bytes(N), 120 * 1024);
    const int warps = g_tune_solve_warps > 0 ? std::min(st->pre_warps, g_tune_solve_warps) : st->pre_warps;
    for (long long c0 = 0; c0 < P.n_in; c0 += st->wg_entries) {
      StateParams Q = P;
      Q.c0 = (int)c0;
      Q.ch = (int)st->wg_entries;
      Q.Wg = st->Wg;
      Q.Ptc16 = st->sh->Ptc16;
      Q.pexp = st->sh->pexp;
      const long long cnt = std::min<long long>(P.n_in - c0, st->wg_entries);  // a bound: the count may be on the device
      const int tiles = (int)((cnt + kAsmRows - 1) / kAsmRows);
      const bool timed = st->time_asm && st->n_aev < csd_state::kAsmEv;
      if (timed) CUDA_TRY(cudaEventRecord(st->aev[2 * st->n_aev], s));
      csd_assemble_tc_kernel<N><<<std::max(1, std::min(tiles, nsm)), 192, asm_smem, s>>>(Q);
      CUDA_TRY(cudaGetLastError());
      if (timed) CUDA_TRY(cudaEventRecord(st->aev[2 * st->n_aev++ + 1], s));
      ++st->asm_launches;
      const int need = (int)std::min<long long>(st->blocks, (cnt + warps - 1) / warps);
      csd_solve_kernel<N, true><<<std::max(need, 1), warps * 32, st->pre_smem, s>>>(Q);
      CUDA_TRY(cudaGetLastError());
    }
    return 0;
  }
  const int warps = g_tune_solve_warps > 0 ? std::min(st->warps, g_tune_solve_warps) : st->warps;
  const int need = (int)std::min<long long>(st->blocks, (P.n_in + warps - 1) / warps);
  csd_solve_kernel<N><<<std::max(need, 1), warps * 32, st->smem, s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_check_launch(csd_state* st, double tol, cudaStream_t s) {
  // one FP64 slot per warp of this grid: at most fp64_slots warps
  using CL = CheckLayout<N>;
  const int wpb = (int)std::min<long long>(CL::WARPS, st->fp64_slots);
  const int blocks = (int)std::max<long long>(1, std::min<long long>(st->fp64_slots / wpb, 65535));
  const int smem = (int)((CL::table_bytes(st->sh->h.nhr) + 15) / 16 * 16) + wpb * CL::WARP;
  CUDA_TRY(cudaFuncSetAttribute(csd_state_check_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  StateParams P = state_params(st);
  csd_state_check_kernel<N><<<blocks, wpb * 32, smem, s>>>(P, st->n, tol, st->chk);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_reuse_launch(csd_state* st, const StateParams& P, cudaStream_t s) {
  const int need = (int)std::min<long long>(st->blocks, (P.n_in + st->reuse_warps - 1) / st->reuse_warps);
  csd_solve_reuse_kernel<N><<<std::max(need, 1), st->reuse_warps * 32, st->reuse_smem, s>>>(P);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
template <int N>
int state_fod_launch(const csd_state* st, float* fod, int64_t fs, uint8_t* so, uint8_t* io, uint32_t* no,
                     cudaStream_t s) {
  const long long tot = st->n * N;
  if (tot == 0) return 0;
  csd_state_fod_kernel<N><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(st->F, st->status, st->iters, st->old,
                                                                        (st->sh->h.nhr + 31) / 32, st->n, fod, fs,
                                                                        so, io, no);
  CUDA_TRY(cudaGetLastError());
  return 0;
}
}  // namespace

#define CSD_DISPATCH(nsh, CALL)                                                          \
  switch (nsh) {                                                                         \
    case 6: { constexpr int NN = 6; CALL; } break;                                       \
    case 15: { constexpr int NN = 15; CALL; } break;                                     \
    case 28: { constexpr int NN = 28; CALL; } break;                                     \
    case 45: { constexpr int NN = 45; CALL; } break;                                     \
    case 66: { constexpr int NN = 66; CALL; } break;                                     \
    case 91: { constexpr int NN = 91; CALL; } break;                                     \
    default: return fail(CSD_ERR_UNSUPPORTED, "unsupported nSH");                        \
  }

extern "C" int csd_state_create(const csd_shared* s, int64_t capacity, csd_state** out) {
  if (!s || !out || capacity <= 0 || capacity > (1LL << 31) - 1)
    return fail(CSD_ERR_INVALID, "csd_state_create: invalid argument");
  *out = nullptr;
  int rc0 = ensure_device(s);
  if (rc0) return rc0;
  std::unique_ptr<csd_state> st(new csd_state);
  st->sh = s;
  st->cap = capacity;
  const int n = s->h.nsh, nw = (s->h.nhr + 31) / 32, HS = s->HS;
  CUDA_TRY(cudaMalloc(&st->F, (size_t)capacity * HS * sizeof(float)));
  CUDA_TRY(cudaMalloc(&st->b, (size_t)capacity * n * sizeof(double)));
  CUDA_TRY(cudaMalloc(&st->old, (size_t)capacity * nw * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&st->old2, (size_t)capacity * nw * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&st->newm, (size_t)capacity * nw * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&st->warm, (size_t)capacity * nw * sizeof(uint32_t)));
  CUDA_TRY(cudaMalloc(&st->slist, (size_t)capacity * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->rlist, (size_t)capacity * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->rcount, (kRunBatch + 1) * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->status, (size_t)capacity));
  CUDA_TRY(cudaMalloc(&st->iters, (size_t)capacity * sizeof(uint16_t)));
  CUDA_TRY(cudaMalloc(&st->cyc, (size_t)capacity * sizeof(uint16_t)));
  CUDA_TRY(cudaMalloc(&st->act[0], (size_t)capacity * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->act[1], (size_t)capacity * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->counter, 2 * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->stats, 4 * sizeof(unsigned long long)));
  CUDA_TRY(cudaMalloc(&st->chk, 2 * sizeof(unsigned long long)));
  CUDA_TRY(cudaMalloc(&st->pcount, (2 * kRunBatch + 2) * sizeof(int)));
  st->async_passes = s->h.niter + 2;
  CUDA_TRY(cudaMalloc(&st->acount, (2 * st->async_passes + 2) * sizeof(int)));
  CUDA_TRY(cudaMalloc(&st->arcount, (st->async_passes + 1) * sizeof(int)));
  for (auto& e : st->ev) CUDA_TRY(cudaEventCreate(&e));
  for (auto& e : st->bev) CUDA_TRY(cudaEventCreate(&e));
  for (auto& e : st->aev) CUDA_TRY(cudaEventCreate(&e));
  int rc = 0;
  CSD_DISPATCH(n, rc = state_shape<NN>(st.get()));
  if (rc) return rc;
  *out = st.release();
  return CSD_OK;
}

extern "C" void csd_state_destroy(csd_state* st) {
  if (!st) return;
  cudaFree(st->F);
  cudaFree(st->b);
  cudaFree(st->old);
  cudaFree(st->old2);
  cudaFree(st->newm);
  cudaFree(st->warm);
  cudaFree(st->slist);
  cudaFree(st->rlist);
  cudaFree(st->rcount);
  cudaFree(st->status);
  cudaFree(st->iters);
  cudaFree(st->cyc);
  cudaFree(st->Lst);
  cudaFree(st->fac);
  cudaFree(st->act[0]);
  cudaFree(st->act[1]);
  cudaFree(st->counter);
  cudaFree(st->stats);
  cudaFree(st->chk);
  cudaFree(st->fp64);
  cudaFree(st->Wg);
  cudaFree(st->pcount);
  cudaFree(st->acount);
  cudaFree(st->arcount);
  for (auto& e : st->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : st->bev)
    if (e) cudaEventDestroy(e);
  for (auto& e : st->aev)
    if (e) cudaEventDestroy(e);
  delete st;
}

extern "C" int csd_state_set(csd_state* st, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                             int64_t volume_stride, const uint8_t* mask, void* stream) {
  if (!st || n_voxels < 0 || n_voxels > st->cap || (n_voxels > 0 && !dwi))
    return fail(CSD_ERR_INVALID, "csd_state_set: invalid argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st->n = n_voxels;
  st->use_warm = 0;
  st->cur = 0;
  st->passes = st->projected = st->solved = 0;
  st->ms_set = st->ms_project = st->ms_solve = st->ms_reuse = 0;
  st->ms_asm = 0;
  st->asm_launches = 0;
  st->launches = 0;
  CUDA_TRY(cudaMemsetAsync(st->counter, 0, sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(st->stats, 0, 4 * sizeof(unsigned long long), s));
  if (n_voxels == 0) {
    st->n_active = 0;
    return CSD_OK;
  }
  StateParams P = state_params(st);
  P.n_in = (int)n_voxels;
  P.dwi = dwi;
  P.vox_stride = voxel_stride;
  P.vol_stride = volume_stride;
  P.mask = mask;
  P.act_out = st->act[0];
  int rc = 0;
  CUDA_TRY(cudaEventRecord(st->ev[0], s));
  CSD_DISPATCH(st->sh->h.nsh, rc = state_set_launch<NN>(st, P, s));
  if (rc) return rc;
  CUDA_TRY(cudaEventRecord(st->ev[1], s));
  int na = 0;
  CUDA_TRY(cudaMemcpyAsync(&na, st->counter, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  float ms = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&ms, st->ev[0], st->ev[1]));
  st->ms_set += ms;
  st->launches += 1;
  st->n_active = na;
  return CSD_OK;
}

extern "C" int csd_state_warm(csd_state* st, const uint32_t* negmask, void* stream) {
  if (!st || !negmask) return fail(CSD_ERR_INVALID, "csd_state_warm: invalid argument");
  const int nw = (st->sh->h.nhr + 31) / 32;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (st->n > 0)
    CUDA_TRY(cudaMemcpyAsync(st->warm, negmask, (size_t)st->n * nw * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  if (g_reuse != 2 && !st->Lst && st->reuse_warps > 0) {
    // storage for the warm sets' factors, on first warm use of the state
    if (cudaMalloc(&st->Lst, (size_t)st->cap * st->lst_floats * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&st->fac, (size_t)st->cap) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(st->Lst);
      st->Lst = nullptr;
      return fail(CSD_ERR_NOMEM, "csd_state_warm: no device memory for the warm-set factors");
    }
  }
  if (st->fac && st->n > 0) CUDA_TRY(cudaMemsetAsync(st->fac, 0, (size_t)st->n, s));
  st->use_warm = 1;
  return CSD_OK;
}

extern "C" int csd_state_reuse_stats(const csd_state* st, double* out) {
  if (!st || !out) return fail(CSD_ERR_INVALID, "csd_state_reuse_stats: invalid argument");
  unsigned long long d[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpy(d, st->stats, sizeof(d), cudaMemcpyDeviceToHost));
  out[0] = (double)d[2];
  out[1] = (double)d[3];
  out[2] = st->ms_reuse;
  return CSD_OK;
}

extern "C" int csd_state_iterate(csd_state* st, int64_t* n_active, void* stream) {
  if (!st) return fail(CSD_ERR_INVALID, "csd_state_iterate: NULL state");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (st->n_active > 0) {
    int rc = 0;
    // pass 1: dense projection of every active voxel -> solve list
    StateParams P = state_params(st);
    P.n_in = (int)st->n_active;
    P.act_in = st->act[st->cur];
    P.act_out = st->slist;
    CUDA_TRY(cudaMemsetAsync(st->counter, 0, 2 * sizeof(int), s));
    CUDA_TRY(cudaEventRecord(st->ev[0], s));
    if (st->use_warm && st->passes == 0) {
      rc = state_warm_first_launch(P, s);  // the first sets are given: nothing to project
    } else {
      CSD_DISPATCH(st->sh->h.nsh, rc = state_project_launch<NN>(st, P, s));
    }
    if (rc) return rc;
    CUDA_TRY(cudaEventRecord(st->ev[1], s));
    int cnt[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(cnt, st->counter, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (cnt[1]) return fail(CSD_ERR_TIMEOUT, "projection: a bounded wait on the tensor cores timed out");
    const int ns = cnt[0];
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, st->ev[0], st->ev[1]));
    st->ms_project += ms;
    st->launches += 1;
    st->projected += st->n_active;
    // pass 2: assemble + factorise the voxels whose set changed -> next active list
    int na = 0;
    if (ns > 0) {
      StateParams Q = state_params(st);
      Q.n_in = ns;
      Q.act_in = st->slist;
      Q.act_out = st->act[st->cur ^ 1];
      CUDA_TRY(cudaMemsetAsync(st->counter, 0, sizeof(int), s));
      CUDA_TRY(cudaEventRecord(st->ev[2], s));
      // later solves of warm-started voxels from their stored factor first
      // (none before the second pass); the full kernel then takes every other
      // voxel (and any the first gave up)
      StateParams Qf = Q;  // the full kernel's input: the solve list, or what the reuse kernel leaves of it
      if (Q.Lst && st->passes > 0) {
        CUDA_TRY(cudaMemsetAsync(st->rcount, 0, sizeof(int), s));
        StateParams Qr = Q;
        Qr.rest_out = st->rlist;
        Qr.n_rest = st->rcount;
        CSD_DISPATCH(st->sh->h.nsh, rc = state_reuse_launch<NN>(st, Qr, s));
        if (rc) return rc;
        st->launches += 1;
        Qf.act_in = st->rlist;
        Qf.n_in_dev = st->rcount;
      }
      CUDA_TRY(cudaEventRecord(st->ev[3], s));
      const long long asm0 = st->asm_launches;
      st->time_asm = true;
      st->n_aev = 0;
      CSD_DISPATCH(st->sh->h.nsh, rc = state_solve_launch<NN>(st, Qf, s));
      st->time_asm = false;
      if (rc) return rc;
      CUDA_TRY(cudaEventRecord(st->ev[1], s));
      int na_err[2] = {0, 0};
      CUDA_TRY(cudaMemcpyAsync(na_err, st->counter, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      CUDA_TRY(cudaStreamSynchronize(s));
      if (na_err[1]) return fail(CSD_ERR_TIMEOUT, "assembly: a bounded wait on the tensor cores timed out");
      na = na_err[0];
      CUDA_TRY(harvest_asm_time(st));
      st->launches += st->asm_launches - asm0;
      float ms2 = 0.f, ms3 = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms2, st->ev[2], st->ev[1]));
      CUDA_TRY(cudaEventElapsedTime(&ms3, st->ev[2], st->ev[3]));
      st->ms_solve += ms2;
      st->ms_reuse += ms3;
      st->launches += 1;
      st->solved += ns;
    }
    st->n_active = na;
    st->cur ^= 1;
    st->passes += 1;
  }
  if (n_active) *n_active = st->n_active;
  return CSD_OK;
}

// Iterate until no voxel is active (or max_passes passes, when > 0).  The
// passes are enqueued in batches of up to kRunBatch without a host round
// trip between them: each kernel reads its input count from the device
// (the count the previous kernel produced) and the launch grids are sized
// for the active count at the start of the batch, an upper bound for every
// later pass since a voxel never becomes active again.  The kernels and
// their per-voxel arithmetic are the ones csd_state_iterate launches, so the
// results are identical to calling csd_state_iterate until it reports 0.
extern "C" int csd_state_run(csd_state* st, int max_passes, int64_t* n_active, void* stream) {
  if (!st) return fail(CSD_ERR_INVALID, "csd_state_run: NULL state");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // batches of 8, then 4, 8, 16 passes: most volumes finish within 8-12
  // passes, so the first batch covers a warm-started run (7 on the benchmark
  // volume) with one host round trip, and the second a plain run's tail
  int done = 0, batch = 8;
  bool first = true;
  while (st->n_active > 0 && (max_passes <= 0 || done < max_passes)) {
    int K = std::min(batch, kRunBatch);
    if (max_passes > 0) K = std::min(K, max_passes - done);
    batch = first ? 4 : 2 * batch;
    first = false;
    const int U = (int)st->n_active;
    CUDA_TRY(cudaMemsetAsync(st->pcount, 0, (2 * K + 1) * sizeof(int), s));
    CUDA_TRY(cudaMemsetAsync(st->rcount, 0, K * sizeof(int), s));
    CUDA_TRY(cudaMemsetAsync(st->counter + 1, 0, sizeof(int), s));
    CUDA_TRY(cudaEventRecord(st->bev[0], s));
    int rc = 0;
    int reuse_launches = 0;
    const long long asm0 = st->asm_launches;
    st->time_asm = true;
    st->n_aev = 0;
    const long long pass0 = st->passes;  // passes since csd_state_set before this batch
    for (int p = 0; p < K; ++p) {
      StateParams P = state_params(st);
      P.n_in = U;  // grid size; the count itself comes from the device after the first pass
      P.n_in_dev = p == 0 ? nullptr : st->pcount + 2 * p;
      P.act_in = st->act[st->cur];
      P.act_out = st->slist;
      P.n_out = st->pcount + 2 * p + 1;
      if (st->use_warm && pass0 + p == 0) {
        rc = state_warm_first_launch(P, s);  // the first sets are given: nothing to project
      } else {
        CSD_DISPATCH(st->sh->h.nsh, rc = state_project_launch<NN>(st, P, s));
      }
      if (rc) return rc;
      CUDA_TRY(cudaEventRecord(st->bev[3 * p + 1], s));
      StateParams Q = state_params(st);
      Q.n_in = U;
      Q.n_in_dev = st->pcount + 2 * p + 1;
      Q.act_in = st->slist;
      Q.act_out = st->act[st->cur ^ 1];
      Q.n_out = st->pcount + 2 * p + 2;
      // later solves of warm-started voxels from their stored factor first
      // (none before the second pass); the full kernel then takes every other
      // voxel (and any the first gave up)
      StateParams Qf = Q;  // the full kernel's input: the solve list, or what the reuse kernel leaves of it
      if (Q.Lst && pass0 + p > 0) {
        ++reuse_launches;
        StateParams Qr = Q;
        Qr.rest_out = st->rlist;
        Qr.n_rest = st->rcount + p;
        CSD_DISPATCH(st->sh->h.nsh, rc = state_reuse_launch<NN>(st, Qr, s));
        if (rc) return rc;
        Qf.act_in = st->rlist;
        Qf.n_in_dev = st->rcount + p;
      }
      CUDA_TRY(cudaEventRecord(st->bev[3 * p + 2], s));
      CSD_DISPATCH(st->sh->h.nsh, rc = state_solve_launch<NN>(st, Qf, s));
      if (rc) return rc;
      CUDA_TRY(cudaEventRecord(st->bev[3 * p + 3], s));
      st->cur ^= 1;
    }
    int cnt[2 * kRunBatch + 1];
    int err = 0;
    CUDA_TRY(cudaMemcpyAsync(cnt, st->pcount, (2 * K + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(&err, st->counter + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    st->time_asm = false;
    if (err) return fail(CSD_ERR_TIMEOUT, "a bounded wait on the tensor cores timed out");
    CUDA_TRY(harvest_asm_time(st));
    cnt[0] = U;
    // every enqueued pass launches its kernels (empty ones return at once)
    st->launches += 2 * K + reuse_launches + (st->asm_launches - asm0);
    for (int p = 0; p < K; ++p) {
      if (cnt[2 * p] == 0) break;
      float a = 0.f, b = 0.f, c = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&a, st->bev[3 * p], st->bev[3 * p + 1]));
      CUDA_TRY(cudaEventElapsedTime(&b, st->bev[3 * p + 1], st->bev[3 * p + 2]));
      CUDA_TRY(cudaEventElapsedTime(&c, st->bev[3 * p + 2], st->bev[3 * p + 3]));
      st->ms_project += a;
      st->ms_reuse += b;
      st->ms_solve += b + c;
      st->projected += cnt[2 * p];
      st->solved += cnt[2 * p + 1];
      st->passes += 1;
      ++done;
    }
    st->n_active = cnt[2 * K];
  }
  if (n_active) *n_active = st->n_active;
  return CSD_OK;
}

// The phased method with no host synchronisation, so that it can be captured
// in a CUDA graph: set() (+ the warm sets), then exactly `passes` passes,
// each kernel reading its voxel count from the device (the grids are sized
// for every voxel; a pass with nothing left returns at once).  A voxel makes
// at most niter + 1 passes, so passes = niter + 1 always reaches the end; the
// results are those of csd_state_set + csd_state_warm + csd_state_run.  With
// warm sets and the factor reuse on, the state's factor storage must exist
// before a capture (csd_state_warm allocates it on first use).  The per-step
// counters of csd_state_stats are not updated; csd_state_async_result
// synchronises and reports the voxels still active and any time-out.
extern "C" int csd_state_run_async(csd_state* st, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                                   int64_t volume_stride, const uint8_t* mask, const uint32_t* warm_negmask,
                                   int passes, void* stream) {
  if (!st || n_voxels < 0 || n_voxels > st->cap || (n_voxels > 0 && !dwi) || passes < 1 ||
      passes > st->async_passes)
    return fail(CSD_ERR_INVALID, "csd_state_run_async: invalid argument (passes must be 1..niter+2)");
  if (warm_negmask && g_reuse != 2 && st->reuse_warps > 0 && !st->Lst)
    return fail(CSD_ERR_INVALID, "csd_state_run_async: call csd_state_warm once first (it allocates the factor storage)");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  st->n = n_voxels;
  st->use_warm = warm_negmask ? 1 : 0;
  st->cur = 0;
  st->n_active = 0;
  st->passes = st->projected = st->solved = 0;
  st->ms_set = st->ms_project = st->ms_solve = st->ms_reuse = 0;
  st->ms_asm = 0;
  st->asm_launches = 0;
  CUDA_TRY(cudaMemsetAsync(st->acount, 0, (2 * passes + 2) * sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(st->arcount, 0, (passes + 1) * sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(st->counter, 0, 2 * sizeof(int), s));
  CUDA_TRY(cudaMemsetAsync(st->stats, 0, 4 * sizeof(unsigned long long), s));
  if (n_voxels == 0) return CSD_OK;
  const int nw = (st->sh->h.nhr + 31) / 32;
  int rc = 0;
  {
    StateParams P = state_params(st);
    P.n_in = (int)n_voxels;
    P.dwi = dwi;
    P.vox_stride = voxel_stride;
    P.vol_stride = volume_stride;
    P.mask = mask;
    P.act_out = st->act[0];
    P.n_out = st->acount;
    CSD_DISPATCH(st->sh->h.nsh, rc = state_set_launch<NN>(st, P, s));
    if (rc) return rc;
  }
  if (warm_negmask) {
    CUDA_TRY(cudaMemcpyAsync(st->warm, warm_negmask, (size_t)n_voxels * nw * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, s));
    if (st->fac) CUDA_TRY(cudaMemsetAsync(st->fac, 0, (size_t)n_voxels, s));
  }
  int cur = 0;
  for (int p = 0; p < passes; ++p) {
    StateParams P = state_params(st);
    P.n_in = (int)n_voxels;  // grid bound; the counts come from the device
    P.n_in_dev = st->acount + 2 * p;
    P.act_in = st->act[cur];
    P.act_out = st->slist;
    P.n_out = st->acount + 2 * p + 1;
    if (warm_negmask && p == 0) {
      rc = state_warm_first_launch(P, s);  // the first sets are given: nothing to project
    } else {
      CSD_DISPATCH(st->sh->h.nsh, rc = state_project_launch<NN>(st, P, s));
    }
    if (rc) return rc;
    StateParams Q = state_params(st);
    Q.n_in = (int)n_voxels;
    Q.n_in_dev = st->acount + 2 * p + 1;
    Q.act_in = st->slist;
    Q.act_out = st->act[cur ^ 1];
    Q.n_out = st->acount + 2 * p + 2;
    StateParams Qf = Q;
    if (Q.Lst && p > 0) {
      StateParams Qr = Q;
      Qr.rest_out = st->rlist;
      Qr.n_rest = st->arcount + p;
      CSD_DISPATCH(st->sh->h.nsh, rc = state_reuse_launch<NN>(st, Qr, s));
      if (rc) return rc;
      Qf.act_in = st->rlist;
      Qf.n_in_dev = st->arcount + p;
    }
    CSD_DISPATCH(st->sh->h.nsh, rc = state_solve_launch<NN>(st, Qf, s));
    if (rc) return rc;
    cur ^= 1;
  }
  st->cur = cur;
  st->async_cur = passes;
  return CSD_OK;
}

// After csd_state_run_async (synchronises the stream): *n_active = voxels
// still iterating after its last pass (0 when it ran enough passes);
// *timed_out = 1 if a bounded wait on the tensor cores gave up.
extern "C" int csd_state_async_result(csd_state* st, int64_t* n_active, int* timed_out, void* stream) {
  if (!st) return fail(CSD_ERR_INVALID, "csd_state_async_result: NULL state");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int cnt = 0, err = 0;
  if (st->async_cur > 0)
    CUDA_TRY(cudaMemcpyAsync(&cnt, st->acount + 2 * st->async_cur, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&err, st->counter + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (n_active) *n_active = cnt;
  if (timed_out) *timed_out = err;
  return CSD_OK;
}

extern "C" int csd_state_stats(const csd_state* st, double* out) {
  if (!st || !out) return fail(CSD_ERR_INVALID, "csd_state_stats: invalid argument");
  unsigned long long d[2] = {0, 0};
  CUDA_TRY(cudaMemcpy(d, st->stats, sizeof(d), cudaMemcpyDeviceToHost));
  out[0] = (double)st->passes;
  out[1] = (double)st->projected;
  out[2] = (double)st->solved;
  out[3] = (double)d[0];
  out[4] = st->ms_set;
  out[5] = st->ms_project;
  out[6] = st->ms_solve;
  out[7] = (double)st->launches;
  return CSD_OK;
}

extern "C" int csd_state_assembly_stats(const csd_state* st, double* out) {
  if (!st || !out) return fail(CSD_ERR_INVALID, "csd_state_assembly_stats: invalid argument");
  out[0] = (double)st->asm_launches;
  out[1] = st->ms_asm;
  out[2] = st->Wg ? (double)st->wg_entries : 0.0;
  return CSD_OK;
}

extern "C" int csd_state_check(csd_state* st, double tol, int64_t* n_checked, int64_t* n_resolved, void* stream) {
  if (!st || !(tol >= 0.0)) return fail(CSD_ERR_INVALID, "csd_state_check: invalid argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  CUDA_TRY(cudaMemsetAsync(st->chk, 0, 2 * sizeof(unsigned long long), s));
  if (st->n > 0) {
    int rc = 0;
    CSD_DISPATCH(st->sh->h.nsh, rc = state_check_launch<NN>(st, tol, s));
    if (rc) return rc;
    st->launches += 1;
  }
  if (n_checked || n_resolved) {
    unsigned long long c[2] = {0, 0};
    CUDA_TRY(cudaMemcpyAsync(c, st->chk, sizeof(c), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    if (n_checked) *n_checked = (int64_t)c[0];
    if (n_resolved) *n_resolved = (int64_t)c[1];
  }
  return CSD_OK;
}

extern "C" int csd_state_fod(const csd_state* st, float* fod, int64_t fod_stride, uint8_t* status,
                             uint8_t* iterations, uint32_t* negmask, void* stream) {
  if (!st || !fod || fod_stride < st->sh->h.nsh) return fail(CSD_ERR_INVALID, "csd_state_fod: invalid argument");
  int rc = 0;
  CSD_DISPATCH(st->sh->h.nsh,
               rc = state_fod_launch<NN>(st, fod, fod_stride, status, iterations, negmask,
                                         static_cast<cudaStream_t>(stream)));
  return rc;
}


// ---------------------------------------------------------------------------
// csd_solve_noalloc: the persistent solve with every piece of device scratch
// (work counter, the scheme's tables, the FP64 fallback slots) carved from
// one file-scope device array instead of cudaMalloc'd workspace.

static constexpr size_t kNoAllocBytes = size_t(24) << 20;  // 24 MiB, held by every device that loads the library
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

static std::mutex g_noalloc_mu;
static std::map<int, unsigned char*> g_noalloc_base;  // device -> device address of g_noalloc_scratch

// Set-up, once per device with that device current: host code may not use
// g_noalloc_scratch's name as an address, so ask the runtime for it.
static int noalloc_base(unsigned char** out) {
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  auto it = g_noalloc_base.find(dev);
  if (it == g_noalloc_base.end()) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(CSD_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                                    cudaGetErrorString(e));
    it = g_noalloc_base.emplace(dev, static_cast<unsigned char*>(p)).first;
  }
  *out = it->second;
  return 0;
}

static size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <int N>
static int noalloc_launch(const csd_shared* s, const csd_volume* v, cudaStream_t st, unsigned char* base) {
  const HostShared& h = s->h;
  // layout: [counter | H32 | H16 | H64 | MtMp | MtM64 | rconvT | M32 | dwis | FP64 slots]
  size_t off = 256;
  const size_t oH32 = off; off = align256(off + s->H32_host.size() * sizeof(float));
  const size_t oH16 = off; off = align256(off + s->H16_host.size() * sizeof(__half));
  const size_t oH64 = off; off = align256(off + h.HR.size() * sizeof(double));
  const size_t oMtMp = off; off = align256(off + s->MtMp_host.size() * sizeof(float));
  const size_t oMtM64 = off; off = align256(off + h.MtM.size() * sizeof(double));
  const size_t oRc = off; off = align256(off + s->rconvT_host.size() * sizeof(float));
  const size_t oM = off; off = align256(off + s->M32_host.size() * sizeof(float));
  const size_t oDw = off; off = align256(off + h.dwis.size() * sizeof(int));
  const size_t oSlots = off;
  if (oSlots >= kNoAllocBytes)
    return fail(CSD_ERR_UNSUPPORTED, "csd_solve_noalloc: the scheme's tables exceed the 24 MiB scratch");
  LaunchShape ls;
  int rc = shape_for<N>(h.nhr, v->n_voxels, &ls);
  if (rc) return rc;
  const size_t per_block = (size_t)ls.warps * Dims<N>::WSZ * sizeof(double);
  const long long fit = (long long)((kNoAllocBytes - oSlots) / per_block);
  if (fit < 1)
    return fail(CSD_ERR_UNSUPPORTED, "csd_solve_noalloc: no room for one block's FP64 slots in the 24 MiB scratch");
  const int blocks = (int)std::min<long long>(ls.blocks, fit);
  CUDA_TRY(cudaMemsetAsync(base, 0, sizeof(unsigned long long), st));
  CUDA_TRY(cudaMemcpyAsync(base + oH32, s->H32_host.data(), s->H32_host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oH16, s->H16_host.data(), s->H16_host.size() * sizeof(__half), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oH64, h.HR.data(), h.HR.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oMtMp, s->MtMp_host.data(), s->MtMp_host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oMtM64, h.MtM.data(), h.MtM.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oRc, s->rconvT_host.data(), s->rconvT_host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oM, s->M32_host.data(), s->M32_host.size() * sizeof(float), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(base + oDw, h.dwis.data(), h.dwis.size() * sizeof(int), cudaMemcpyHostToDevice, st));
  SolveParams P;
  std::memset(&P, 0, sizeof(P));
  P.n_vol = 1;
  P.nhr = h.nhr;
  P.nw = (h.nhr + 31) / 32;
  P.refine = refine_of(s);
  P.fast_cycles = g_fast_cycles == 1;
  P.cond_thr = (float)s->cond_thr;
  P.total = v->n_voxels;
  P.queue = reinterpret_cast<unsigned long long*>(base);
  P.fp64_scratch = reinterpret_cast<double*>(base + oSlots);
  VolumeDesc& d = P.vol[0];
  d.sc.H32 = reinterpret_cast<const float*>(base + oH32);
  d.sc.H16 = reinterpret_cast<const __half*>(base + oH16);
  d.sc.H64 = reinterpret_cast<const double*>(base + oH64);
  d.sc.MtMp = reinterpret_cast<const float*>(base + oMtMp);
  d.sc.MtM64 = reinterpret_cast<const double*>(base + oMtM64);
  d.sc.rconvT = reinterpret_cast<const float*>(base + oRc);
  d.sc.M32 = reinterpret_cast<const float*>(base + oM);
  d.sc.dwis = reinterpret_cast<const int*>(base + oDw);
  d.sc.ndw = h.ndw;
  d.sc.ninit = h.ninit;
  d.sc.niter = h.niter;
  d.sc.threshold = (float)h.threshold;
  d.sc.hscale = pow2f(s->hexp);
  d.dwi = v->dwi;
  d.n_voxels = v->n_voxels;
  d.vox_stride = v->voxel_stride;
  d.vol_stride = v->volume_stride;
  d.first = 0;
  d.mask = v->mask;
  d.warm = v->warm_negmask;
  d.fod = v->fod;
  d.fod_stride = v->fod_stride;
  d.status = v->status;
  d.iters = v->iterations;
  d.negmask = v->negmask;
  return launch_persistent<N>(P, ls.smem, ls.warps, blocks, st);
}

extern "C" int csd_solve_noalloc(const csd_shared* s, const csd_volume* v, void* stream) {
  if (!s || !v) return fail(CSD_ERR_INVALID, "csd_solve_noalloc: NULL argument");
  if (v->n_voxels < 0) return fail(CSD_ERR_INVALID, "csd_solve_noalloc: negative voxel count");
  if (v->n_voxels == 0) return CSD_OK;
  if (!v->dwi || !v->fod) return fail(CSD_ERR_INVALID, "csd_solve_noalloc: NULL dwi or fod");
  if (v->fod_stride < s->h.nsh) return fail(CSD_ERR_INVALID, "csd_solve_noalloc: fod_stride smaller than nSH");
  if (v->voxel_stride < 0 || v->volume_stride < 0) return fail(CSD_ERR_INVALID, "csd_solve_noalloc: negative stride");
  unsigned char* base = nullptr;
  int rc = noalloc_base(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CSD_DISPATCH(s->h.nsh, rc = noalloc_launch<NN>(s, v, st, base));
  return rc;
}


// ---------------------------------------------------------------------------
// csd_dwi2fod_host_phased: the phased method (optionally warm-started by the
// network) on HOST buffers.  The volume is cut into slabs; each slab's
// host->device copy, solve and device->host copy run on one of two streams,
// so the copies of one slab overlap the passes of the other.

namespace {
constexpr int kHostBufs = 8;  // buffer sets (and streams): slabs in flight at once
constexpr int kHostConcDefault = 1 << 20;  // slabs computing at once by default (all)
// passes enqueued per slab when every slab has its own state: the benchmark
// volume needs 7 (warm) / 10 (plain); a slab with voxels still active after
// them is finished by csd_state_run (same iteration) after one host sync,
// instead of enqueueing niter + 2 passes whose empty launches cost ~40 us each
constexpr int kHostAsyncPasses = 16;
struct PhasedHostWS {
  uint64_t sh_id = 0;  // the csd_shared the states were made for (ids are never reused; addresses can be)
  int64_t cap = 0;
  int nbuf = 0;  // buffer sets allocated (each with its stream)
  csd_state* st[kHostBufs] = {};
  float* dwi[kHostBufs] = {};
  float* fod[kHostBufs] = {};
  uint8_t* small[kHostBufs] = {};   // mask | status | iterations
  uint32_t* warm[kHostBufs] = {};
  cudaStream_t stream[kHostBufs] = {};
  int* hres = nullptr;  // pinned: per slab, voxels still active after its passes and the timed-out flag
  int64_t hres_cap = 0;
  uint8_t* hsi = nullptr;  // pinned staging of status and iterations (2 x voxels), copied out at the end
  int64_t hsi_cap = 0;
  cudaEvent_t cev[16] = {};  // per slab: its compute is done (orders the next slabs' compute)
};
std::mutex g_phws_mu;
std::map<int, PhasedHostWS> g_phws;

void release(PhasedHostWS& w) {
  for (int i = 0; i < kHostBufs; ++i) {
    csd_state_destroy(w.st[i]);
    cudaFree(w.dwi[i]);
    cudaFree(w.fod[i]);
    cudaFree(w.small[i]);
    cudaFree(w.warm[i]);
    w.st[i] = nullptr;
    w.dwi[i] = w.fod[i] = nullptr;
    w.small[i] = nullptr;
    w.warm[i] = nullptr;
  }
  cudaFreeHost(w.hres);
  w.hres = nullptr;
  w.hres_cap = 0;
  cudaFreeHost(w.hsi);
  w.hsi = nullptr;
  w.hsi_cap = 0;
  w.nbuf = 0;
  w.cap = 0;
  w.sh_id = 0;
}
}  // namespace

extern "C" int csd_dwi2fod_host_phased(const csd_shared* s, csd_mlp* net, const float* dwi, int64_t n_voxels,
                                       const uint8_t* mask, float* fod, uint8_t* status, uint8_t* iterations) {
  if (!s || n_voxels < 0 || (n_voxels > 0 && (!dwi || !fod)))
    return fail(CSD_ERR_INVALID, "csd_dwi2fod_host_phased: invalid argument");
  if (n_voxels == 0) return CSD_OK;
  int dev = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  int rc0 = ensure_device(s);
  if (rc0) return rc0;
  std::lock_guard<std::mutex> lk(g_phws_mu);
  PhasedHostWS& w = g_phws[dev];
  const int nvol = s->h.nvol, nsh = s->h.nsh, nw = (s->h.nhr + 31) / 32;
  const int64_t nslab = std::min<int64_t>(g_host_slabs > 0 ? g_host_slabs : 8, std::max<int64_t>(1, n_voxels / 131072));
  const int64_t per = (n_voxels + nslab - 1) / nslab;
  const bool async = g_host_async != 2;
  // the asynchronous path gives every slab (up to kHostBufs) its own buffers
  // and stream, so that all uploads can run ahead; the host-driven one
  // alternates two
  const int nb = async ? (int)std::max<int64_t>(2, std::min<int64_t>(nslab, kHostBufs)) : 2;
  if (w.sh_id != s->id || w.cap < per || w.nbuf < nb) {
    release(w);
    for (int i = 0; i < nb; ++i) {
      int rc = csd_state_create(s, per, &w.st[i]);
      if (rc) return rc;
      CUDA_TRY(cudaMalloc(&w.dwi[i], (size_t)per * nvol * sizeof(float)));
      CUDA_TRY(cudaMalloc(&w.fod[i], (size_t)per * nsh * sizeof(float)));
      CUDA_TRY(cudaMalloc(&w.small[i], (size_t)per * 3));
      CUDA_TRY(cudaMalloc(&w.warm[i], (size_t)per * nw * sizeof(uint32_t)));
      if (!w.stream[i]) {
        // earlier slabs at higher priority: they finish first, so their
        // downloads overlap the later slabs' compute, which fills the SMs
        // the earlier ones leave idle in their tail passes
        int lo = 0, hi = 0;
        CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        const int levels = lo - hi + 1;
        const int prio = hi + std::min(levels - 1, i * levels / kHostBufs);
        CUDA_TRY(cudaStreamCreateWithPriority(&w.stream[i], cudaStreamNonBlocking, prio));
      }
    }
    w.sh_id = s->id;
    w.cap = per;
    w.nbuf = nb;
  }
  auto upload = [&](int64_t k) -> int {
    const int64_t a = k * per, n = std::min(per, n_voxels - a);
    const int b = (int)(k % nb);
    CUDA_TRY(cudaMemcpyAsync(w.dwi[b], dwi + a * nvol, (size_t)n * nvol * sizeof(float), cudaMemcpyHostToDevice,
                             w.stream[b]));
    if (mask) CUDA_TRY(cudaMemcpyAsync(w.small[b], mask + a, (size_t)n, cudaMemcpyHostToDevice, w.stream[b]));
    return 0;
  };
  int rc = 0;
  if (async) {
    // every slab enqueued at once, slab k on stream k % nb with that
    // stream's buffers (the stream orders their reuse): upload, inference,
    // the phased run as csd_state_run_async's fixed passes (niter + 2, so
    // complete; a pass with nothing left returns at once), FODs, download.
    // One slab's tail of nearly empty passes then overlaps the other's work.
    if (w.hres_cap < nslab) {
      cudaFreeHost(w.hres);
      w.hres = nullptr;
      w.hres_cap = 0;
      CUDA_TRY(cudaMallocHost(&w.hres, (size_t)nslab * 2 * sizeof(int)));
      w.hres_cap = nslab;
    }
    // status and iterations go through pinned staging: a copy into pageable
    // memory would hold the host until that slab is done
    if ((status || iterations) && w.hsi_cap < n_voxels) {
      cudaFreeHost(w.hsi);
      w.hsi = nullptr;
      w.hsi_cap = 0;
      CUDA_TRY(cudaMallocHost(&w.hsi, (size_t)n_voxels * 2));
      w.hsi_cap = n_voxels;
    }
    if (net)
      for (int i = 0; i < nb; ++i)  // the warm-set factor storage, once
        if (!w.st[i]->Lst && (rc = csd_state_warm(w.st[i], w.warm[i], w.stream[i]))) return rc;
    const int64_t conc = g_host_conc > 0 ? g_host_conc : kHostConcDefault;
    // fewer passes than niter + 2 only when no state is reused by a later slab
    int host_passes = kHostAsyncPasses;
    if (const char* env = std::getenv("CSD_HOST_PASSES")) {  // fewer, to exercise the finishing path in tests
      const int v = std::atoi(env);
      if (v >= 1) host_passes = v;
    }
    auto passes0 = [&](const csd_state* S) { return nslab <= nb ? std::min(S->async_passes, host_passes)
                                                                : S->async_passes; };
    for (auto& e : w.cev)
      if (!e) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int64_t k = 0; k < nslab; ++k) {
      const int64_t a = k * per, n = std::min(per, n_voxels - a);
      if (n <= 0) break;
      const int b = (int)(k % nb);
      cudaStream_t st = w.stream[b];
      csd_state* S = w.st[b];
      if ((rc = upload(k))) return rc;
      // the upload above runs ahead; the compute waits for slab k - conc's
      if (conc < nslab && k >= conc) CUDA_TRY(cudaStreamWaitEvent(st, w.cev[k - conc], 0));
      const uint8_t* dmask = mask ? w.small[b] : nullptr;
      if (net && (rc = csd_mlp_predict(net, w.dwi[b], n, nvol, 1, dmask, 0.f, w.warm[b], st))) return rc;
      if ((rc = csd_state_run_async(S, w.dwi[b], n, nvol, 1, dmask, net ? w.warm[b] : nullptr, passes0(S), st)))
        return rc;
      uint8_t* dst = w.small[b] + per;
      uint8_t* dit = w.small[b] + 2 * per;
      if ((rc = csd_state_fod(S, w.fod[b], nsh, status ? dst : nullptr, iterations ? dit : nullptr, nullptr, st)))
        return rc;
      CUDA_TRY(cudaEventRecord(w.cev[k], st));
      CUDA_TRY(cudaMemcpyAsync(w.hres + 2 * k, S->acount + 2 * S->async_cur, sizeof(int), cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaMemcpyAsync(w.hres + 2 * k + 1, S->counter + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
      if (status) CUDA_TRY(cudaMemcpyAsync(w.hsi + a, dst, (size_t)n, cudaMemcpyDeviceToHost, st));
      if (iterations) CUDA_TRY(cudaMemcpyAsync(w.hsi + n_voxels + a, dit, (size_t)n, cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaMemcpyAsync(fod + a * nsh, w.fod[b], (size_t)n * nsh * sizeof(float), cudaMemcpyDeviceToHost, st));
    }
    for (int i = 0; i < nb; ++i) CUDA_TRY(cudaStreamSynchronize(w.stream[i]));
    bool finished = false;
    for (int64_t k = 0; k < nslab && k * per < n_voxels; ++k) {
      if (w.hres[2 * k + 1]) return fail(CSD_ERR_TIMEOUT, "csd_dwi2fod_host_phased: a bounded wait timed out");
      if (!w.hres[2 * k]) continue;
      const int b = (int)(k % nb);
      csd_state* S = w.st[b];
      if (nslab > nb || passes0(S) >= S->async_passes)
        return fail(CSD_ERR_CUDA, "csd_dwi2fod_host_phased: voxels left iterating after niter + 2 passes");
      // voxels still iterating after the enqueued passes: the rest of the
      // iteration by csd_state_run on the same state, then this slab's
      // outputs again
      const int64_t a = k * per, n = std::min(per, n_voxels - a);
      cudaStream_t st = w.stream[b];
      S->n_active = w.hres[2 * k];
      S->passes = passes0(S);
      if ((rc = csd_state_run(S, 0, nullptr, st))) return rc;
      uint8_t* dst = w.small[b] + per;
      uint8_t* dit = w.small[b] + 2 * per;
      if ((rc = csd_state_fod(S, w.fod[b], nsh, status ? dst : nullptr, iterations ? dit : nullptr, nullptr, st)))
        return rc;
      if (status) CUDA_TRY(cudaMemcpyAsync(w.hsi + a, dst, (size_t)n, cudaMemcpyDeviceToHost, st));
      if (iterations) CUDA_TRY(cudaMemcpyAsync(w.hsi + n_voxels + a, dit, (size_t)n, cudaMemcpyDeviceToHost, st));
      CUDA_TRY(cudaMemcpyAsync(fod + a * nsh, w.fod[b], (size_t)n * nsh * sizeof(float), cudaMemcpyDeviceToHost, st));
      finished = true;
    }
    if (finished)
      for (int i = 0; i < nb; ++i) CUDA_TRY(cudaStreamSynchronize(w.stream[i]));
    if (status) std::memcpy(status, w.hsi, (size_t)n_voxels);
    if (iterations) std::memcpy(iterations, w.hsi + n_voxels, (size_t)n_voxels);
    return CSD_OK;
  }
  // host round trips: enqueue the first slab's upload, then per slab:
  // enqueue the next upload on the other stream, solve this slab, enqueue
  // its download
  rc = upload(0);
  if (rc) return rc;
  for (int64_t k = 0; k < nslab; ++k) {
    const int64_t a = k * per, n = std::min(per, n_voxels - a);
    if (n <= 0) break;
    const int b = (int)(k & 1);
    cudaStream_t st = w.stream[b];
    if (k + 1 < nslab && (k + 1) * per < n_voxels) {
      // the other buffer's previous download must finish before reuse
      CUDA_TRY(cudaStreamSynchronize(w.stream[b ^ 1]));
      if ((rc = upload(k + 1))) return rc;
    }
    const uint8_t* dmask = mask ? w.small[b] : nullptr;
    if ((rc = csd_state_set(w.st[b], w.dwi[b], n, nvol, 1, dmask, st))) return rc;
    if (net) {
      if ((rc = csd_mlp_predict(net, w.dwi[b], n, nvol, 1, dmask, 0.f, w.warm[b], st))) return rc;
      if ((rc = csd_state_warm(w.st[b], w.warm[b], st))) return rc;
    }
    if ((rc = csd_state_run(w.st[b], 0, nullptr, st))) return rc;
    uint8_t* dst = w.small[b] + per;
    uint8_t* dit = w.small[b] + 2 * per;
    if ((rc = csd_state_fod(w.st[b], w.fod[b], nsh, status ? dst : nullptr, iterations ? dit : nullptr, nullptr, st)))
      return rc;
    CUDA_TRY(cudaMemcpyAsync(fod + a * nsh, w.fod[b], (size_t)n * nsh * sizeof(float), cudaMemcpyDeviceToHost, st));
    if (status) CUDA_TRY(cudaMemcpyAsync(status + a, dst, (size_t)n, cudaMemcpyDeviceToHost, st));
    if (iterations) CUDA_TRY(cudaMemcpyAsync(iterations + a, dit, (size_t)n, cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(cudaStreamSynchronize(w.stream[0]));
  CUDA_TRY(cudaStreamSynchronize(w.stream[1]));
  return CSD_OK;
}

#include "hr_dirs_builtin.inc"
