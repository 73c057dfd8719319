/*
 * csd_b200.h -- C ABI of the B200-native single-shell constrained spherical
 * deconvolution (CSD) library, libcsd_b200.so.
 *
 * It replaces the hot path of MRtrix3's `dwi2fod csd`:
 *   MR::DWI::SDeconv::CSD::Shared (src/dwi/sdeconv/csd.h:46-212) -> csd_shared_*
 *   MR::DWI::SDeconv::CSD set/iterate/FOD (csd.h:221-271)         -> csd_state_*
 *   the ThreadedLoop over voxels in cmd/dwi2fod.cpp:275-281
 *     with CSD_Processor (cmd/dwi2fod.cpp:120-176)                -> csd_solve,
 *                                                                    csd_dwi2fod_host
 * and, for the commands around it:
 *   sh2peaks (cmd/sh2peaks.cpp)                                   -> csd_sh2peaks
 *   amp2sh (cmd/amp2sh.cpp)                                       -> csd_amp2sh[_rician]
 *   Math::ICLS (core/math/constrained_least_squares.h), the solver
 *     of dwi2fod msmt_csd and amp2response                        -> csd_icls_*
 *   amp2response's accumulation (cmd/amp2response.cpp)            -> csd_amp2response_accumulate
 *   dwi2tensor + tensor2metric -fa -vector                        -> csd_dwi2tensor
 *   FMLS::Segmenter (src/dwi/fmls.cpp), fod2fixel's segmentation  -> csd_fmls_*
 * Plain pointers and sizes only.  Device pointers are CUDA global memory on
 * the current device; a `stream` argument is a cudaStream_t (NULL = legacy
 * default stream).  All functions return 0 on success or a negative CSD_ERR_*
 * code; csd_last_error() then describes the failure (thread-local).
 */
#ifndef CSD_B200_H
#define CSD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSD_OK 0
#define CSD_ERR_INVALID (-1)     /* invalid argument (the reference throws MR::Exception) */
#define CSD_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define CSD_ERR_TIMEOUT (-3)     /* a bounded device wait gave up */
#define CSD_ERR_NOMEM (-4)       /* device allocation failed */
#define CSD_ERR_UNSUPPORTED (-5) /* e.g. lmax above the compiled maximum */

/* Per-voxel status byte (low nibble = outcome, high bits = flags).  The
 * reference reports non-convergence only as an INFO log
 * (cmd/dwi2fod.cpp:142-144) and never checks the LLT status (csd.h:264). */
#define CSD_STATUS_MASKED 0       /* outside the mask: FOD written as zeros (dwi2fod.cpp:130-133) */
#define CSD_STATUS_CONVERGED 1    /* iterate() returned true within niter */
#define CSD_STATUS_NITER 2        /* niter iterate() calls without convergence */
#define CSD_STATUS_NONFINITE 3    /* a non-finite sample: FOD zeros (dwi2fod.cpp:166-167) */
#define CSD_STATUS_FP64 0x10      /* flag: a factorisation was redone in FP64 */
#define CSD_STATUS_CHOLFAIL 0x20  /* flag: the normal matrix was not positive definite */
#define CSD_STATUS_WARM_RESTART 0x40 /* flag: warm start abandoned, re-solved from the plain start */

#define CSD_MAX_LMAX 12           /* largest lmax compiled (91 coefficients) */

/* Options of `dwi2fod csd` (src/dwi/sdeconv/csd.cpp:318-346,
 * cmd/dwi2fod.cpp:38-59) and the two config-file keys the path reads. */
typedef struct csd_params {
  int lmax;                 /* -lmax; 0 = min(lmax of response, 8) (csd.h:127) */
  int niter;                /* -niter, default 50 (csd.h:35) */
  double neg_lambda;        /* -neg_lambda, default 1 (csd.h:32) */
  double norm_lambda;       /* -norm_lambda, default 1 (csd.h:33) */
  double threshold;         /* -threshold, default 0 (csd.h:34) */
  const double* filter;     /* -filter (NULL = [1 1 1], csd.h:136-137) */
  int n_filter;
  double bzero_threshold;   /* config BZeroThreshold, default 10 (dwi/gradient.cpp:92-95) */
  double bvalue_epsilon;    /* config BValueEpsilon, default 80 (dwi/shells.cpp:43-46) */
  double fp64_condition;    /* GPU only: condition estimate above which a voxel's
                               factorisation is redone in FP64 (default 1e6) */
  int refine;               /* GPU only: one FP64-residual refinement step of the FP32
                               solution -- 0 never, 1 after every solve, 2 once at the
                               fixed point (then re-checked), 3 (default) only for voxels
                               whose negative set cycles in FP32, after every solve */
  const double* shells;     /* -shells b-values (dwi/shells.cpp:100-239 with
                               select_shells(true, false, true), csd.h:64): exactly
                               one non-b=0 shell must match, and no b=0 shell;
                               NULL / 0 = the largest b-value shell */
  int n_shells;
} csd_params;

typedef struct csd_shared csd_shared;  /* immutable after creation, like CSD::Shared after init() */

/* Fill *p with the reference defaults. */
void csd_params_init(csd_params* p);

/* CSD::Shared(header) + parse_cmdline_options() + set_response() + init()
 * (csd.h:52-198).  grad: [n_volumes][4] host doubles (x y z b), as
 * DWI::get_DW_scheme reads them (dwi/gradient.cpp:280).  response: zonal SH
 * coefficients l=0,2,..  hr_dirs: [n_hr][2] azimuth/elevation, or NULL for
 * the built-in 300 directions (csd.h:54, -directions at csd.h:84-86).
 * Uploads the tables to the current device. */
int csd_shared_create(const csd_params* p, const double* grad, int n_volumes, const double* response,
                      int n_response, const double* hr_dirs, int n_hr, csd_shared** out);
void csd_shared_destroy(csd_shared* s);

/* CSD::Shared::nSH() (csd.h:200-202). */
int csd_shared_nsh(const csd_shared* s);
/* info[8] = lmax, lmax_response, lmax_data, nSH, n_init, n_dw, n_hr, niter */
int csd_shared_info(const csd_shared* s, int* info);
/* The `dwis` member (csd.h:62): volume indices of the selected shell [n_dw]. */
int csd_shared_dwis(const csd_shared* s, int* out);
/* Host FP64 copies of the public matrices: which = 0 rconv [n_init][n_dw],
 * 1 M [n_dw][nSH], 2 Mt_M [nSH][nSH] (symmetric, with norm_lambda),
 * 3 HR_trans [n_hr][nSH], 4 scalars [threshold, norm_lambda, neg_lambda]. */
int csd_shared_matrix(const csd_shared* s, int which, double* out);

/* One image to deconvolve.  dwi[v*voxel_stride + t*volume_stride] is volume
 * t of voxel v (float32, the layout `with_direct_io(3)` gives when
 * voxel_stride = n_volumes and volume_stride = 1, dwi2fod.cpp:279).
 * All pointers are device pointers; optional ones may be NULL. */
typedef struct csd_volume {
  const float* dwi;
  int64_t n_voxels;
  int64_t voxel_stride;
  int64_t volume_stride;
  const uint8_t* mask;            /* optional [n_voxels], 0 = skip (dwi2fod.cpp:158-162) */
  const uint32_t* warm_negmask;   /* optional [n_voxels][ceil(n_hr/32)] first negative set */
  float* fod;                     /* [n_voxels][fod_stride] output, first nSH used */
  int64_t fod_stride;
  uint8_t* status;                /* optional [n_voxels] CSD_STATUS_* */
  uint8_t* iterations;            /* optional [n_voxels] iterate() calls (saturates at 255) */
  uint32_t* negmask;              /* optional [n_voxels][ceil(n_hr/32)] final negative set */
} csd_volume;

/* Deconvolve n_volumes images in ONE persistent launch: volumes[i] uses
 * shared[i] (each may have its own gradient scheme, but all must share nSH
 * and n_hr).  Warps pull voxels from a device work queue; converged voxels
 * free their warp for the next.  Equivalent to running CSD_Processor over
 * every voxel (dwi2fod.cpp:128-147).  Asynchronous on `stream`. */
int csd_solve(const csd_shared* const* shared, const csd_volume* volumes, int n_volumes, void* stream);

/* End-to-end call on HOST buffers: dwi [n_voxels][n_volumes] float32,
 * voxel-interleaved; mask optional; fod [n_voxels][nSH].  Stages through
 * pinned memory in slabs with copies overlapped with the solve.  Synchronous. */
int csd_dwi2fod_host(const csd_shared* s, const float* dwi, int64_t n_voxels, const uint8_t* mask,
                     float* fod, uint8_t* status, uint8_t* iterations);

typedef struct csd_mlp csd_mlp;  /* the warm-start network, below */

/* The phased method on HOST buffers (same layout as csd_dwi2fod_host):
 * per slab of voxels, csd_state_set, then -- when `net` is not NULL -- the
 * network's predicted first negative sets (csd_mlp_predict + csd_state_warm),
 * then the passes until no voxel is active, then csd_state_fod.  The slabs
 * (at most 8 by default, knob 8) each get their own buffers and stream and
 * are all enqueued at once, so the uploads run ahead and one slab's copies
 * and tail passes overlap the others' work: each slab's passes are
 * csd_state_run_async's, 16 of them (niter + 2 when slabs share buffers),
 * and a slab with voxels still iterating after them is finished by
 * csd_state_run on its own state after one host synchronisation (the same
 * iteration, so the same outputs).  Knob 11 = 2 drives each slab with
 * csd_state_run instead; knob 13 > 0 makes slab k's compute wait for slab
 * k - knob's.  Synchronous; CSD_ERR_TIMEOUT if a bounded device wait gave
 * up. */
int csd_dwi2fod_host_phased(const csd_shared* s, csd_mlp* net, const float* dwi, int64_t n_voxels,
                            const uint8_t* mask, float* fod, uint8_t* status, uint8_t* iterations);

/* ---- per-step surface: CSD::set / iterate / FOD (csd.h:237-271) over a
 *      batch of voxels (the reference object is one voxel: a batch of 1).
 *      The plain GPU method drives these phases from the host, one pass per
 *      iterate(): projection of all still-active voxels, compaction, then
 *      assembly + factorisation of the voxels whose negative set changed. */
typedef struct csd_state csd_state;
int csd_state_create(const csd_shared* s, int64_t capacity, csd_state** out);
void csd_state_destroy(csd_state* st);
/* CSD::set for n_voxels voxels (clamps <0 to 0; non-finite or masked voxels
 * are marked done with a zero FOD).  Resets the iteration state. */
int csd_state_set(csd_state* st, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                  int64_t volume_stride, const uint8_t* mask, void* stream);
/* Replace the first negative set of every active voxel (warm start). */
int csd_state_warm(csd_state* st, const uint32_t* negmask, void* stream);
/* One CSD::iterate() on every active voxel.  *n_active receives how many
 * voxels are still iterating afterwards (synchronises the stream). */
int csd_state_iterate(csd_state* st, int64_t* n_active, void* stream);
/* CSD::iterate() until every voxel is done (the `for (n < niter) if
 * (iterate()) break;` loop of dwi2fod.cpp:137-139 over the batch), or for at most max_passes passes when
 * max_passes > 0.  Passes are enqueued in batches that read their voxel
 * counts on the device, with one host round trip per batch; the results are
 * identical to calling csd_state_iterate until it reports 0.  *n_active (may
 * be NULL) receives how many voxels are still iterating (synchronises). */
int csd_state_run(csd_state* st, int max_passes, int64_t* n_active, void* stream);
/* csd_state_set + (csd_state_warm when warm_negmask is not NULL) +
 * csd_state_run as exactly `passes` passes with no host synchronisation,
 * so that the whole method can be captured in a CUDA graph (several states
 * on several streams: many volumes, each with its own scheme, in one graph
 * launch).  Every kernel reads its voxel count from the device; a pass with
 * nothing left returns at once, so passes = niter + 1 always reaches the end
 * (at most niter + 2).  The results equal the synchronous calls'.  With warm
 * sets, call csd_state_warm on the state once before a capture (it
 * allocates the factor storage).  csd_state_stats is not updated. */
int csd_state_run_async(csd_state* st, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                        int64_t volume_stride, const uint8_t* mask, const uint32_t* warm_negmask, int passes,
                        void* stream);
/* After csd_state_run_async (synchronises): voxels still iterating after its
 * last pass (0 once it ran enough passes) and whether a bounded wait timed out. */
int csd_state_async_result(csd_state* st, int64_t* n_active, int* timed_out, void* stream);
/* Work and device time since the last csd_state_set: out[8] = passes, voxels
 * projected, voxels solved, sum of |negative set| over the solves that
 * assembled their system (not those of csd_state_reuse_stats), then the
 * device milliseconds of the set / projection / solve kernels (the solve
 * time includes the reuse kernel's), and the number of kernel launches. */
int csd_state_stats(const csd_state* st, double* out);
/* Factor reuse of a warm-started state since the last csd_state_set: out[3]
 * = solves that went through the warm set's stored Cholesky factor (a
 * Woodbury correction by the directions added to / dropped from the warm set,
 * at most 16; more, a voxel whose set cycles, or a first solve that needed
 * FP64 take the full assembly + factorisation), the sum of those changed-
 * direction counts, and the device milliseconds of that kernel.  No
 * counterpart in the reference: the iteration and its sets are csd.h:245-269's,
 * only the arithmetic of each later W^-1 b differs.  csd_state_warm allocates
 * the factor storage (capacity x ~4.8 KB at lmax 8) on a state's first warm use. */
int csd_state_reuse_stats(const csd_state* st, double* out);
/* The phased solve's rank-k assembly (csd.h:255-262) on the tensor cores
 * since the last csd_state_set: out[3] = launches of the assembly kernel
 * (csd_assemble_tc_kernel: W = Mt_M + H[S]^T H[S] of 128 listed voxels at a
 * time as the product of their 0/1 set masks with a table of HR_trans
 * products, FP16 hi + lo, FP32 accumulation in tensor memory), their device
 * milliseconds (recorded by csd_state_iterate / csd_state_run only; the
 * solve time of csd_state_stats includes it), and how many systems one
 * launch holds (the solve list runs in chunks of that many; 0: the
 * assembly runs inside the solve kernel on mma.sync, as for more than 320
 * constraint directions or launch knob 12 = 1). */
int csd_state_assembly_stats(const csd_state* st, double* out);
/* FP64 check of every finished voxel (converged or at niter): the residual
 * r = b - (Mt_M + HR_trans[S]^T HR_trans[S]) F of the voxel's final set S
 * (csd.h:255-264) in FP64; a voxel with max|r| > tol max|b| has its system
 * re-assembled and solved in FP64 (status gains CSD_STATUS_FP64); tol 0
 * re-solves every finished voxel.
 * *n_checked / *n_resolved (may be NULL; otherwise the call synchronises)
 * receive the counts.  No counterpart in the reference, which solves in
 * FP64 throughout. */
int csd_state_check(csd_state* st, double tol, int64_t* n_checked, int64_t* n_resolved, void* stream);
/* CSD::FOD(): copy F (float) out, plus optional status/iterations/negmask. */
int csd_state_fod(const csd_state* st, float* fod, int64_t fod_stride, uint8_t* status,
                  uint8_t* iterations, uint32_t* negmask, void* stream);

/* Allocation-free variant of csd_solve for one volume.  No counterpart in
 * the reference: it exists for callers that must not call cudaMalloc while
 * they run -- applications whose own allocator owns all device memory, or
 * services whose memory footprint has to stay fixed after start-up -- so
 * every piece of device scratch the solve needs (its work counter, the
 * scheme's tables, the FP64 fallback slots) lives in one 24 MiB array of
 * static device memory that every device which loads the library holds
 * until exit.  The caller still owns dwi / mask / fod / status buffers.
 * The first call on a device looks up that array's device address (set-up,
 * once per device); make that first call before any stream capture.  Each
 * call copies the scheme's tables into the array and zeroes the counter, so
 * calls overlapping on the GPU (other streams, other threads) race: run them
 * one at a time per device.  Returns CSD_ERR_UNSUPPORTED if the scheme's
 * tables plus one block's FP64 slots do not fit; grids shrink to fit. */
int csd_solve_noalloc(const csd_shared* s, const csd_volume* volume, void* stream);

/* ---- warm-start network.  No counterpart in the reference: a 66 -> 256 ->
 *      256 -> 300 MLP (GELU, sigmoid head; BF16 weights and activations, FP32
 *      accumulation and Adam) that predicts each voxel's converged negative
 *      set from its normalised signal.  The prediction only replaces the
 *      first negative set (csd_volume.warm_negmask); the iteration then runs
 *      to its own stopping rule, and a voxel that does not reach a fixed
 *      point is re-solved from the plain start. */
int csd_mlp_create(int n_in, int n_hidden, int n_out, uint64_t seed, csd_mlp** out);
void csd_mlp_destroy(csd_mlp* m);
int64_t csd_mlp_param_count(const csd_mlp* m);
/* flat FP32 parameters [W1 b1 W2 b2 W3 b3], weights [out][in padded to 16 / 8] */
int csd_mlp_get_params(const csd_mlp* m, float* out, int64_t n);
int csd_mlp_set_params(csd_mlp* m, const float* in, int64_t n);
/* input = (S_t / mean over b0_index of S - mean_t) / stdev_t for every volume t */
int csd_mlp_set_inputs(csd_mlp* m, const int* b0_index, int n_b0, const float* mean, const float* stdev);
/* normalised BF16 inputs [n][n_in padded to 16] for training (device) */
int csd_mlp_inputs(const csd_mlp* m, const float* dwi, int64_t n_voxels, int64_t voxel_stride,
                   int64_t volume_stride, uint16_t* x, void* stream);
/* one epoch of Adam over n rows in batches (a multiple of 128) of shuffled order */
int csd_mlp_train_epoch(csd_mlp* m, const uint16_t* x, const uint32_t* negmask, int64_t n, int batch, float lr,
                        float weight_decay, uint64_t seed, float* mean_loss, void* stream);
/* predicted first negative sets [n][ceil(n_out/32)] (device): direction d is in
 * the set when its logit exceeds logit_threshold (0 = probability 1/2);
 * masked-out voxels get none */
int csd_mlp_predict(csd_mlp* m, const float* dwi, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                    const uint8_t* mask, float logit_threshold, uint32_t* negmask, void* stream);
/* checks: BCE gradients (host copy of the flat gradient) and raw logits [n][n_out padded to 8] */
int csd_mlp_gradients(csd_mlp* m, const uint16_t* x, const uint32_t* negmask, int64_t n, float* grad_out,
                      float* loss_out);
int csd_mlp_logits(csd_mlp* m, const uint16_t* x, int64_t n, float* z_out);

/* ---- sh2peaks (cmd/sh2peaks.cpp:99-303, core/math/SH.h:515-650) on device
 *      buffers: for each voxel's SH coefficients (float, [n][voxel_stride],
 *      lmax even, 2..12) a Newton search from every seed direction (n_seeds
 *      [azimuth elevation] pairs in radians, at most 256; the reference's 60
 *      are mrtrix3_b200/data/sh2peaks_seeds_60.txt), duplicates within
 *      |cos| > 0.99 of an earlier peak and peaks below `threshold` dropped;
 *      output [n][3 npeaks] amplitude-scaled directions, NaN-padded (npeaks
 *      at most 16).  With n_directions = npeaks unit vectors (-direction), or
 *      a per-voxel [n][3 npeaks] peaks_in (-peaks), each output is the peak
 *      of largest |cos| with its target; else the largest peaks.  Masked,
 *      non-finite and all-isotropic voxels give NaN (check_input).  Returns
 *      without synchronising. */
int csd_sh2peaks(const float* sh, int64_t n_voxels, int64_t voxel_stride, int lmax, const uint8_t* mask,
                 const float* seeds_azel, int n_seeds, int npeaks, float threshold, const float* directions,
                 int n_directions, const float* peaks_in, float* peaks_out, void* stream);

/* ---- amp2sh (cmd/amp2sh.cpp:108-127, 153-171) on device buffers: per voxel
 *      of `amp` ([n][voxel_stride], volumes volume_stride apart) the SH
 *      coefficients fit * a in FP64, a = the amplitudes of the nd volumes
 *      `dwis`, scaled by nb0 / (1 + their b=0 sum) when `normalise` (b=0
 *      volumes `bzeros`); fit = pinv(SH2amp) [nsh][nd] (double), nd <= 800
 *      (CSD_ERR_INVALID beyond).  All arrays
 *      are device pointers; output float [n][out_stride].  The volume
 *      indices in `dwis` and `bzeros` must address volumes of the voxel (the
 *      kernel reads them unchecked; the Python binding checks them).  Returns
 *      without synchronising.  The -rician correction: csd_amp2sh_rician. */
int csd_amp2sh(const float* amp, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride, const double* fit,
               int nsh, const int* dwis, int nd, const int* bzeros, int nb0, int normalise, float* sh_out,
               int64_t out_stride, void* stream);

/* ---- amp2sh -rician (cmd/amp2sh.cpp:129-150, 180-197): csd_amp2sh's fit
 *      reweighted for the Rician noise bias, up to 20 rounds per voxel, FP64;
 *      sh2amp [nd][nsh] (double, device) is the SH-to-amplitude mapping whose
 *      pinv is `fit`; noise: device float per voxel (noise[v * noise_stride]).
 *      nsh <= 153.  Returns without synchronising. */
int csd_amp2sh_rician(const float* amp, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                      const double* fit, const double* sh2amp, int nsh, const int* dwis, int nd, const int* bzeros,
                      int nb0, int normalise, const float* noise, int64_t noise_stride, float* sh_out,
                      int64_t out_stride, void* stream);

/* ---- amp2response (cmd/amp2response.cpp:152-190): accumulate, over the
 *      voxels of `mask` (device uint8 [n] or NULL = all), the normal
 *      equations of one shell's zonal response fit: M += T^T T (lower
 *      triangle of [nz][nz], nz = lmax/2 + 1, lmax even <= 12) and b += T^T a,
 *      T_i the normalised zonal Legendre values at the elevation of volume
 *      `volumes[i]`'s direction `dirs[i]` ([n_dirs][3] device doubles) from the
 *      voxel's fibre direction (fibre_dir[v * dir_stride + c * dir_comp_stride],
 *      c = x y z, device float), folded into [0, pi/2]; a the amplitudes
 *      (amp[v * voxel_stride + volumes[i] * volume_stride]).  M and b are
 *      device doubles, added to (zero them first).  FP64.  Returns without
 *      synchronising. */
int csd_amp2response_accumulate(const float* amp, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                                const float* fibre_dir, int64_t dir_stride, int64_t dir_comp_stride,
                                const uint8_t* mask, const double* dirs, int n_dirs, const int* volumes, int lmax,
                                double* M, double* b, void* stream);

/* ---- dwi2tensor (cmd/dwi2tensor.cpp:106-135) with tensor2metric's FA and
 *      principal eigenvector (cmd/tensor2metric.cpp:156-247), as dwi2response's
 *      fa / manual algorithms use them: per voxel of dwi ([n][voxel_stride],
 *      volumes volume_stride apart, device float) the iteratively reweighted
 *      log-linear fit (iter reweightings, default 2; ols: unweighted start)
 *      with bmat = -grad2bmatrix (device double [n_volumes][7], rows [-b gx^2,
 *      -b gy^2, -b gz^2, -2b gx gy, -2b gx gz, -2b gy gz, 1]), FP64.  Outputs
 *      (device float): dt [n][dt_stride] = Dxx Dyy Dzz Dxy Dxz Dyz; b0 [n],
 *      fa [n] and vec [n][3] (the principal eigenvector times FA) or NULL.
 *      Voxels outside `mask` (device uint8 or NULL) give zeros.  Returns
 *      without synchronising. */
int csd_dwi2tensor(const float* dwi, int64_t n_voxels, int64_t voxel_stride, int64_t volume_stride,
                   const double* bmat, int n_volumes, const uint8_t* mask, int iter, int ols, float* dt,
                   int64_t dt_stride, float* b0, float* fa, float* vec, void* stream);

/* ---- inequality-constrained least squares, batched: the solver of
 *      dwi2fod msmt_csd (src/dwi/sdeconv/msmt_csd.h:249-270) and of
 *      Math::ICLS (core/math/constrained_least_squares.h).
 *
 * csd_icls_create replaces ICLS::Problem (constrained_least_squares.h:
 * 90-151): min ||H x - b||^2 subject to A x >= t, the last num_eq rows of
 * A as equalities; H [nmeas][nparam], A [ncons][nparam] row-major host FP64,
 * t [ncons] or NULL (zeros); solution_reg scales the largest diagonal entry
 * of H^T H added to its diagonal, constraint_reg is added to the diagonal of
 * the active-set systems (nparam <= 256, ncons <= 4096, nmeas <= 4096, num_eq
 * <= 512); max_niter 0 = 10 nparam; tol the violation below
 * -tol that activates a constraint.  Set-up in FP64 on the host, tables
 * uploaded to the current device.  Errors: CSD_ERR_INVALID (sizes, H^T H not
 * positive definite, a zero constraint row).
 *
 * csd_icls_solve replaces ICLS::Solver::operator() (:241-370) for n
 * right-hand sides b (device float, [n][voxel_stride], measurements
 * meas_stride apart), FP64 inside: x (device float [n][x_stride], x_stride
 * >= nparam), niter (device int32 [n] or NULL: the solver's rounds; -1 where
 * an active set outgrew 512 rows, with x NaN), pred (device float [n]
 * [pred_stride] or NULL: the predicted measurements H x, dwi2fod msmt_csd's
 * -predicted_signal).  mask (device uint8 [n] or NULL): 0 skips the voxel
 * (x = 0, pred = 0).  A non-finite b gives x = NaN.  Returns without
 * synchronising; grows a per-warp scratch buffer on first use. */
typedef struct csd_icls csd_icls;
int csd_icls_create(const double* H, int nmeas, int nparam, const double* A, int ncons, const double* t,
                    int num_eq, double solution_reg, double constraint_reg, int max_niter, double tol,
                    csd_icls** out);
void csd_icls_destroy(csd_icls* problem);
/* The problem already in standard form (constrained_least_squares.h:67-70,
 * 124-126, 139-140): HtH [nparam][nparam] (host, its lower triangle read) is
 * H^T H, and the right-hand sides given to the solver are H^T b (nmeas =
 * nparam).  As amp2response's constrained fit (amp2response.cpp:345-346). */
int csd_icls_create_standard(const double* HtH, int nparam, const double* A, int ncons, const double* t,
                             int num_eq, double solution_reg, double constraint_reg, int max_niter, double tol,
                             csd_icls** out);
/* out4 = {nmeas, nparam, ncons, max_niter} */
int csd_icls_info(const csd_icls* problem, int* out4);
int csd_icls_solve(csd_icls* problem, const float* b, int64_t n, int64_t voxel_stride, int64_t meas_stride,
                   const uint8_t* mask, float* x, int64_t x_stride, int32_t* niter, float* pred,
                   int64_t pred_stride, void* stream);
/* csd_icls_solve with FP64 right-hand sides and solutions (device
 * pointers; no mask, no predicted measurements). */
int csd_icls_solve_f64(csd_icls* problem, const double* b, int64_t n, int64_t voxel_stride, int64_t meas_stride,
                       double* x, int64_t x_stride, int32_t* niter, void* stream);
/* csd_icls_solve on HOST buffers: b [n][voxel_stride] float (measurements
 * contiguous), mask [n] or NULL, x [n][nparam], niter [n] or NULL, pred
 * [n][nmeas] or NULL.  Stages through device memory kept with the problem
 * (grown as needed, freed by csd_icls_destroy); synchronous.  Calls on one
 * problem must not overlap. */
int csd_icls_solve_host(csd_icls* problem, const float* b, int64_t n, int64_t voxel_stride, const uint8_t* mask,
                        float* x, int32_t* niter, float* pred);

/* Launch-shape knobs (process-wide), chosen by the project's autotuner
 * (mrtrix3_b200/autotune.py): which = 0 warps per block of the persistent
 * kernel, 1 warps per block of the phased solve kernel, 2 projection blocks
 * per SM, 3 projection kernel of the phased method (1 mma.sync, 2 tcgen05
 * with the accumulators in tensor memory; up to 320 constraint directions),
 * 4 phased solve kernel (1 a warp per voxel, 2 / 3 groups of 16 / 8 lanes
 * per voxel, lmax <= 8), 5 phased set kernel (1 a warp per voxel, 2 tiles
 * of 64 voxels), 6 csd_mlp_predict kernels (1 one GEMM per layer, 2 the
 * fused tcgen05 kernel; 66..80 -> 256 -> 256 -> <=320 networks); value 0 =
 * built-in default, 7 the jump of exactly periodic two-cycles to their
 * last call (1 on, 2 off; by default on in the phased method, off in the
 * persistent kernel), 8 the most slabs csd_dwi2fod_host_phased cuts a volume
 * into (0 = 8), 9 the csd_amp2sh kernel (1 a dot product a thread, 2 FP64
 * FMA tiles, 3 FP64 tensor cores where they apply: nd <= 64, nSH <= 48;
 * 0 = the fastest that applies), 10 the warm-started phased method's later
 * solves from the warm set's stored factor (0 default = 1 on, 2 off), 11
 * csd_dwi2fod_host_phased enqueueing every slab's passes at once with no
 * host round trips (0 default = 1 on, 2 off: one round trip per batch), 12
 * the phased solve's rank-k assembly (0 default = 2, 1 mma.sync inside the
 * solve kernel, 2 tcgen05 ahead of it, up to 320 constraint directions;
 * the grouped solve kernels of knob 4 always assemble with mma.sync), 13
 * csd_dwi2fod_host_phased's slabs computing at once (0 default = all; k:
 * slab j's compute waits for slab j - k's).
 * Knobs 0-5, 7, 8, 11 and 13 leave the outputs unchanged bit for bit; knob 6 changes
 * the FP32 summation order of the logits, knob 9 the FP64 summation order of
 * the coefficients, knob 10 the FP32 arithmetic of the later solves, knob
 * 12 the FP32 summation order of the assembled systems (same iteration,
 * results within the parity tolerance). */
int csd_set_launch_config(int which, int value);

/* ---- fod2fixel's FMLS FOD segmenter (src/dwi/fmls.cpp:118-311,
 *      cmd/fod2fixel.cpp).
 *
 * csd_fmls_tables carries what Segmenter's constructor (fmls.cpp:118-140)
 * builds, as host arrays: the ndir unit directions [ndir][3] (the 1281-
 * direction set), their neighbour lists (adj_off [ndir + 1] into adj,
 * at most 16 a direction), the integration weights [ndir], the SH ->
 * amplitude matrix [ndir][nsh] of lmax (<= 16), SH::PrecomputedAL's table
 * [al_ndir][n_al] at elevations n al_inc, FastLookupSet's grid (num_az x
 * num_el cells from az_begin / el_begin in steps az_step / el_step, cell c
 * listing grid[grid_off[c] .. grid_off[c + 1])), and the lobe thresholds
 * (-fmls_integral, -fmls_peak_value, -fmls_lobe_merge_ratio). */
typedef struct csd_fmls_tables {
  int ndir, lmax, nsh;
  const double* unit;
  const double* weight;
  const int32_t* adj_off;
  const int32_t* adj;
  int n_adj;
  const double* sh2amp;
  int al_ndir, n_al;
  double al_inc;
  const double* al;
  int num_az, num_el;
  double az_begin, el_begin, az_step, el_step;
  const int32_t* grid_off;
  const int32_t* grid;
  int n_grid;
  double integral_threshold, peak_value_threshold, merge_ratio;
} csd_fmls_tables;

/* csd_fmls_create replaces FMLS::Segmenter's constructor: checks the tables
 * and copies them to the current device.  Errors: CSD_ERR_INVALID. */
typedef struct csd_fmls csd_fmls;
int csd_fmls_create(const csd_fmls_tables* tables, csd_fmls** out);
/* csd_fmls_create_default: the same on the built-in 1281-direction set (its
 * hull adjacency and integration weights compiled in; the SH transform,
 * Legendre table and lookup grid built on the host), as fod2fixel's
 * Segmenter (dirs (1281), lmax) with load_fmls_thresholds' values.
 * Errors: CSD_ERR_INVALID (lmax odd, negative or above 16). */
int csd_fmls_create_default(int lmax, double integral_threshold, double peak_value_threshold, double merge_ratio,
                            csd_fmls** out);
void csd_fmls_destroy(csd_fmls* segmenter);

/* csd_fmls_segment replaces Segmenter::operator() (fmls.cpp:159-311) for n
 * voxels of SH coefficients (device float [n][voxel_stride], coefficients
 * coef_stride apart; FP64 inside).  counts (device int32 [n]): the number of
 * lobes kept in each voxel (0 where mask, device uint8 [n] or NULL, is 0);
 * fixels (device float [n][max_fixels][8]): per lobe, in the reference's
 * order, the unit mean direction (3), the direction of the largest peak
 * (3), the integral (AFD) and the largest peak amplitude; only the first
 * max_fixels lobes of a voxel are written, so a count above max_fixels asks
 * for another pass with more room.  A voxel with a non-finite coefficient
 * has no lobes.  Returns without synchronising; grows a per-warp scratch
 * buffer on first use, and on first use allocates the state of one round of
 * 16,384 voxels (about 230 MB for the 1281 directions; the voxels go in
 * rounds of three launches).  Calls on one segmenter share those buffers:
 * run them on one stream, or use one segmenter per stream. */
int csd_fmls_segment(csd_fmls* segmenter, const float* fod, int64_t n_voxels, int64_t voxel_stride,
                     int64_t coef_stride, const uint8_t* mask, int max_fixels, int32_t* counts, float* fixels,
                     void* stream);

/* Thread-local description of the last failure. */
const char* csd_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* CSD_B200_H */
