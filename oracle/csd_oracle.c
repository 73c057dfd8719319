/*
 * csd_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of MRtrix3's single-shell constrained spherical
 * deconvolution (`dwi2fod csd`, MR::DWI::SDeconv::CSD, src/dwi/sdeconv/csd.h).
 * It is the checker the CUDA path is compared against, and the CPU baseline
 * that bench.py times ("port": the reference itself needs Eigen, which is not
 * present, so it cannot be compiled here).  Nothing in the product library
 * links, loads or calls this file.
 *
 * Parity pinning: the reference ships no golden vectors for this path (its
 * test_data submodule is absent), so this restatement is pinned by
 *   - the reference's own Legendre recursion (core/math/legendre.h) compiled
 *     from its source by oracle/build_ref.sh and compared bit-for-bit,
 *   - an independent numpy/scipy implementation (tests/test_oracle.py),
 *   - known-answer tests (SH orthonormality, single-fibre peak, niter=0).
 * The end-to-end CSD output itself is "parity unpinned" against reference-run
 * data.
 *
 * Every function cites the reference lines it follows.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_MAX_L 30

/* ---- core/math/SH.h:46-73 ---------------------------------------------- */
static int sh_NforL(int lmax) { return (lmax + 1) * (lmax + 2) / 2; }
static int sh_index(int l, int m) { return l * (l + 1) / 2 + m; }
/* SH.h:70-73: LforN evaluates sqrt in single precision (float(1+8N)). */
static int sh_LforN(int N) {
  if (!N) return 0;
  return 2 * (int)floor((sqrtf((float)(1 + 8 * N)) - 3.0) / 4.0);
}
/* ZSH.h:42-57 */
static int zsh_NforL(int lmax) { return 1 + lmax / 2; }
static int zsh_LforN(int N) { return 2 * (N - 1); }

/* ---- core/math/legendre.h:66-70 (helper) -------------------------------- */
static double plm_sph_helper(double x, double m) {
  return (m < 1.0 ? 1.0 : x * (m - 1.0) / m * plm_sph_helper(x, m - 2.0));
}

/* ---- core/math/legendre.h:101-123: normalised associated Legendre array --- */
void oracle_plm_sph(double *array, int lmax, int m, double x) {
  double x2 = x * x;
  if (m && x2 >= 1.0) {
    for (int n = m; n <= lmax; ++n) array[n] = 0.0;
    return;
  }
  array[m] = 0.282094791773878;
  if (m) array[m] *= sqrt((double)(2 * m + 1) * plm_sph_helper(1.0 - x2, 2.0 * m));
  if (m & 1) array[m] = -array[m];
  if (lmax == m) return;
  double f = sqrt((double)(2 * m + 3));
  array[m + 1] = x * f * array[m];
  for (int n = m + 2; n <= lmax; n++) {
    array[n] = x * array[n - 1] - array[n - 2] / f;
    f = sqrt((double)(4 * n * n - 1) / (double)(n * n - m * m));
    array[n] *= f;
  }
}

/* ---- core/math/SH.h:82-104: SH -> amplitude transform, [ndir x NforL] ---- */
void oracle_init_transform(const double *dirs, int ndir, int lmax, double *SHT) {
  const int N = sh_NforL(lmax);
  const double sqrt2 = 1.41421356237309504880;
  double AL[ORACLE_MAX_L + 1];
  for (int i = 0; i < ndir; i++) {
    double *row = SHT + (size_t)i * N;
    for (int c = 0; c < N; c++) row[c] = 0.0;
    const double az = dirs[2 * i], el = dirs[2 * i + 1];
    const double z = cos(el);
    oracle_plm_sph(AL, lmax, 0, z);
    for (int l = 0; l <= lmax; l += 2) row[sh_index(l, 0)] = AL[l];
    for (int m = 1; m <= lmax; m++) {
      oracle_plm_sph(AL, lmax, m, z);
      for (int l = ((m & 1) ? m + 1 : m); l <= lmax; l += 2) {
        row[sh_index(l, m)] = sqrt2 * AL[l] * cos(m * az);
        row[sh_index(l, -m)] = sqrt2 * AL[l] * sin(m * az);
      }
    }
  }
}

/* ---- plain Cholesky (lower), stands in for Eigen's LLT/LDLT --------------
 * Eigen's blocked LLT (csd.h:264) and pivoted LDLT (least_squares.h:42)
 * differ from this unblocked factorisation only by rounding (~1e-15 rel). */
static int chol_lower(double *A, int n) {
  for (int j = 0; j < n; j++) {
    double d = A[j * n + j];
    for (int k = 0; k < j; k++) d -= A[j * n + k] * A[j * n + k];
    if (!(d > 0.0)) return -1;
    d = sqrt(d);
    A[j * n + j] = d;
    for (int i = j + 1; i < n; i++) {
      double s = A[i * n + j];
      for (int k = 0; k < j; k++) s -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = s / d;
    }
  }
  return 0;
}
static void chol_solve(const double *L, int n, double *x) {
  for (int i = 0; i < n; i++) {
    double s = x[i];
    for (int k = 0; k < i; k++) s -= L[i * n + k] * x[k];
    x[i] = s / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = x[i];
    for (int k = i + 1; k < n; k++) s -= L[k * n + i] * x[k];
    x[i] = s / L[i * n + i];
  }
}

/* ---- shared state: the public members of CSD::Shared (csd.h:204-211) ----- */
typedef struct oracle_shared {
  int lmax, lmax_response, lmax_data, n, nr, ndw, nhr, niter, nvol;
  double neg_lambda, norm_lambda, threshold;
  int *dwis;        /* [ndw] volume indices of the selected shell */
  double *DW_dirs;  /* [ndw][2] az, el */
  double *rconv;    /* [nr][ndw] */
  double *M;        /* [ndw][n] */
  double *MtM;      /* [n][n], lower triangle valid, diagonal has norm_lambda */
  double *HR;       /* [nhr][n] HR_trans (scaled) */
} oracle_shared;

static void set_err(char *err, int errlen, const char *msg) {
  if (err && errlen > 0) {
    strncpy(err, msg, (size_t)errlen - 1);
    err[errlen - 1] = 0;
  }
}

/* ---- core/dwi/shells.cpp:300-411: b-value clustering ---------------------- */
static void region_query(const double *b, int nvol, double bval, double b0thr, double eps,
                         int *idx, int *nidx) {
  for (int i = 0; i < nvol; i++)
    if (b[i] > b0thr && fabs(bval - b[i]) < eps) idx[(*nidx)++] = i;
}

/* Returns the volume indices of the largest non-b=0 shell, i.e.
 * Shells(grad).select_shells(true,false,true).largest().get_volumes()
 * (csd.h:62-64) without a -shells option.  Returns count or <0 on error. */
static int select_largest_shell(const double *b, int nvol, double b0thr, double eps, int *out,
                                char *err, int errlen) {
  int *clusters = calloc((size_t)nvol, sizeof(int));
  char *visited = calloc((size_t)nvol, 1);
  int *nb = malloc(sizeof(int) * (size_t)nvol * (size_t)nvol * 2 + 16);
  int *nb2 = malloc(sizeof(int) * (size_t)nvol + 16);
  int clusterIdx = 0;
  for (int ii = 0; ii < nvol; ii++)
    if (b[ii] <= b0thr) {
      visited[ii] = 1;
      clusterIdx = 1;
      clusters[ii] = 1;
    }
  for (int ii = 0; ii < nvol; ii++) {
    if (visited[ii]) continue;
    visited[ii] = 1;
    int nn = 0;
    region_query(b, nvol, b[ii], b0thr, eps, nb, &nn);
    if (b[ii] > b0thr && nn < 3) {
      clusters[ii] = 0;
    } else {
      clusters[ii] = ++clusterIdx;
      for (int i = 0; i < nn; i++) {
        if (!visited[nb[i]]) {
          visited[nb[i]] = 1;
          int nn2 = 0;
          region_query(b, nvol, b[nb[i]], b0thr, eps, nb2, &nn2);
          if (nn2 >= 3)
            for (int j = 0; j < nn2; j++) nb[nn++] = nb2[j];
        }
        if (clusters[nb[i]] == 0) clusters[nb[i]] = clusterIdx;
      }
    }
  }
  int num_shells = clusterIdx, ret = -1;
  if (num_shells < 1 || num_shells > sqrt((double)nvol)) {
    set_err(err, errlen, "DWI volumes could not be classified into b-value shells");
    goto done;
  }
  /* shells.cpp:311-322 + sort by mean (:339): pick the shell of largest mean */
  {
    double best_mean = -1.0;
    int best = -1, nshell = 0, has_b0 = 0;
    double smallest_mean = 1e300;
    for (int s = 1; s <= num_shells; s++) {
      double mean = 0.0;
      int cnt = 0;
      for (int v = 0; v < nvol; v++)
        if (clusters[v] == s) {
          mean += b[v];
          cnt++;
        }
      if (!cnt) continue;
      nshell++;
      mean /= cnt;
      if (mean < smallest_mean) smallest_mean = mean;
      if (mean > best_mean) {
        best_mean = mean;
        best = s;
      }
    }
    has_b0 = smallest_mean <= b0thr;
    /* shells.cpp:235-241: single non-zero shell required, else keep largest */
    if (nshell == 1 && has_b0) {
      set_err(err, errlen, "No non b=0 data found, but the command requires a non b=0 shell");
      goto done;
    }
    if (best_mean <= b0thr) {
      set_err(err, errlen, "no non-b=0 shell");
      goto done;
    }
    int cnt = 0;
    for (int v = 0; v < nvol; v++)
      if (clusters[v] == best) out[cnt++] = v;
    ret = cnt;
  }
done:
  free(clusters);
  free(visited);
  free(nb);
  free(nb2);
  return ret;
}

/* ---- CSD::Shared ctor + init (csd.h:52-68, 117-198) ---------------------- */
int oracle_shared_init(const double *grad_in, int nvol, const double *response, int nresp,
                       const double *hr_dirs, int nhr, int lmax_cmdline, const double *filter,
                       int nfilter, double neg_lambda, double norm_lambda, double threshold,
                       int niter, double b0thr, double bval_eps, oracle_shared **out, char *err,
                       int errlen) {
  *out = NULL;
  if (nvol <= 0 || nhr <= 0 || nresp <= 0) {
    set_err(err, errlen, "invalid sizes");
    return -1;
  }
  /* gradient.cpp:286-310: normalise directions, scale b by |g|^2 if needed */
  double *grad = malloc(sizeof(double) * 4 * (size_t)nvol);
  memcpy(grad, grad_in, sizeof(double) * 4 * (size_t)nvol);
  double maxlog = 0.0;
  double *sq = malloc(sizeof(double) * (size_t)nvol);
  for (int r = 0; r < nvol; r++) {
    double *g = grad + 4 * r;
    sq[r] = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (sq[r]) {
      double s = sqrt(sq[r]);
      g[0] /= s;
      g[1] /= s;
      g[2] /= s;
    }
    double lg = sq[r] > 0.0 ? fabs(log(sq[r])) : 0.0;
    if (lg > maxlog) maxlog = lg;
  }
  if (maxlog > 0.01)
    for (int r = 0; r < nvol; r++) grad[4 * r + 3] *= sq[r];
  free(sq);

  double *bvals = malloc(sizeof(double) * (size_t)nvol);
  for (int r = 0; r < nvol; r++) bvals[r] = grad[4 * r + 3];
  int *dwis = malloc(sizeof(int) * (size_t)nvol);
  int ndw = select_largest_shell(bvals, nvol, b0thr, bval_eps, dwis, err, errlen);
  free(bvals);
  if (ndw < 0) {
    free(grad);
    free(dwis);
    return -1;
  }
  /* gradient.h:77-95: az = atan2(y,x), el = acos(z/|g|) */
  double *DW_dirs = malloc(sizeof(double) * 2 * (size_t)ndw);
  for (int i = 0; i < ndw; i++) {
    const double *g = grad + 4 * dwis[i];
    DW_dirs[2 * i] = atan2(g[1], g[0]);
    double z = g[2] / sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    DW_dirs[2 * i + 1] = z >= 1.0 ? 0.0 : (z <= -1.0 ? M_PI : acos(z));
  }
  free(grad);

  int lmax_data = sh_LforN(ndw);             /* csd.h:67 */
  int lmax_response = zsh_LforN(nresp);      /* csd.h:112 */
  if (lmax_data <= 0) {                      /* csd.h:121-122 */
    set_err(err, errlen, "data contain too few directions even for lmax = 2");
    free(dwis);
    free(DW_dirs);
    return -1;
  }
  if (lmax_response <= 0) {                  /* csd.h:124-125 */
    set_err(err, errlen, "response function does not contain anisotropic terms");
    free(dwis);
    free(DW_dirs);
    return -1;
  }
  int lmax = lmax_cmdline ? lmax_cmdline : (lmax_response < 8 ? lmax_response : 8); /* :127 */
  if (lmax <= 0 || lmax % 2 || lmax > ORACLE_MAX_L) {
    set_err(err, errlen, "lmax must be a positive even integer");
    free(dwis);
    free(DW_dirs);
    return -1;
  }
  int t = lmax_data < lmax ? lmax_data : lmax;       /* csd.h:133 */
  lmax_response = lmax_response < t ? lmax_response : t;

  /* csd.h:136-138: init_filter default [1,1,1], resized to NforL(lmax_response) */
  int nfilt = zsh_NforL(lmax_response);
  double *filt = calloc((size_t)nfilt, sizeof(double));
  if (filter && nfilter > 0) {
    for (int i = 0; i < nfilt && i < nfilter; i++) filt[i] = filter[i];
  } else {
    for (int i = 0; i < nfilt && i < 3; i++) filt[i] = 1.0;
  }
  /* csd.h:140-142 + ZSH.h:221-231: RH = response / Y_l0(0), zero-padded */
  int nRH = zsh_NforL(lmax) > nresp ? zsh_NforL(lmax) : nresp;
  double *RH = calloc((size_t)nRH, sizeof(double));
  {
    int lr = zsh_LforN(nresp);
    double AL[2 * ORACLE_MAX_L + 3];
    oracle_plm_sph(AL, lr, 0, 1.0);
    for (int l = 0; l <= lr; l += 2) RH[l / 2] = response[l / 2] / AL[l];
  }

  /* csd.h:145-158: rconv = pinv(fconv + 1e-2 on the (non-square) diagonal) */
  int nr = sh_NforL(lmax_response);
  double *fconv = malloc(sizeof(double) * (size_t)ndw * nr);
  oracle_init_transform(DW_dirs, ndw, lmax_response, fconv);
  for (int i = 0; i < ndw && i < nr; i++) fconv[i * nr + i] += 1.0e-2;
  double *rconv = malloc(sizeof(double) * (size_t)nr * ndw);
  {
    /* least_squares.h:41-42: (F^T F)^-1 F^T (rows >= cols in practice) */
    if (ndw < nr) {
      set_err(err, errlen, "fewer DW directions than init coefficients");
      free(filt); free(RH); free(fconv); free(rconv); free(dwis); free(DW_dirs);
      return -1;
    }
    double *FtF = calloc((size_t)nr * nr, sizeof(double));
    for (int i = 0; i < nr; i++)
      for (int j = 0; j < nr; j++) {
        double s = 0.0;
        for (int k = 0; k < ndw; k++) s += fconv[k * nr + i] * fconv[k * nr + j];
        FtF[i * nr + j] = s;
      }
    if (chol_lower(FtF, nr)) {
      set_err(err, errlen, "pinv: F^T F not positive definite");
      free(FtF); free(filt); free(RH); free(fconv); free(rconv); free(dwis); free(DW_dirs);
      return -1;
    }
    double *col = malloc(sizeof(double) * (size_t)nr);
    for (int k = 0; k < ndw; k++) {
      for (int i = 0; i < nr; i++) col[i] = fconv[k * nr + i];
      chol_solve(FtF, nr, col);
      for (int i = 0; i < nr; i++) rconv[i * ndw + k] = col[i];
    }
    free(col);
    free(FtF);
  }
  {
    int l = 0, nl = 1;
    for (int row = 0; row < nr; row++) {
      if (row >= nl) {
        l++;
        nl = sh_NforL(2 * l);
      }
      double s = filt[l] / RH[l];
      for (int k = 0; k < ndw; k++) rconv[row * ndw + k] *= s;
    }
  }
  free(fconv);
  free(filt);

  /* csd.h:163-172: forward convolution, columns scaled by RH[l] */
  int n = sh_NforL(lmax);
  double *M = malloc(sizeof(double) * (size_t)ndw * n);
  oracle_init_transform(DW_dirs, ndw, lmax, M);
  {
    int l = 0, nl = 1;
    for (int c = 0; c < n; c++) {
      if (c >= nl) {
        l++;
        nl = sh_NforL(2 * l);
      }
      for (int k = 0; k < ndw; k++) M[k * n + c] *= RH[l];
    }
  }
  free(RH);

  /* csd.h:175-180: HR_trans scaled by neg_lambda*50*response[0]/nhr */
  double *HR = malloc(sizeof(double) * (size_t)nhr * n);
  oracle_init_transform(hr_dirs, nhr, lmax, HR);
  double cm = neg_lambda * 50.0 * response[0] / (double)nhr;
  for (size_t i = 0; i < (size_t)nhr * n; i++) HR[i] *= cm;
  threshold *= cm;

  /* csd.h:184-195: Mt_M lower, plus norm_lambda on the diagonal */
  double *MtM = calloc((size_t)n * n, sizeof(double));
  for (int i = 0; i < n; i++)
    for (int j = 0; j <= i; j++) {
      double s = 0.0;
      for (int k = 0; k < ndw; k++) s += M[k * n + i] * M[k * n + j];
      MtM[i * n + j] = s;
    }
  if (norm_lambda) {
    norm_lambda *= 0.0002 * MtM[0];
    for (int i = 0; i < n; i++) MtM[i * n + i] += norm_lambda;
  }

  oracle_shared *sh = calloc(1, sizeof(oracle_shared));
  sh->lmax = lmax;
  sh->lmax_response = lmax_response;
  sh->lmax_data = lmax_data;
  sh->n = n;
  sh->nr = nr;
  sh->ndw = ndw;
  sh->nhr = nhr;
  sh->niter = niter;
  sh->nvol = nvol;
  sh->neg_lambda = neg_lambda;
  sh->norm_lambda = norm_lambda;
  sh->threshold = threshold;
  sh->dwis = dwis;
  sh->DW_dirs = DW_dirs;
  sh->rconv = rconv;
  sh->M = M;
  sh->MtM = MtM;
  sh->HR = HR;
  *out = sh;
  return 0;
}

void oracle_shared_free(oracle_shared *sh) {
  if (!sh) return;
  free(sh->dwis);
  free(sh->DW_dirs);
  free(sh->rconv);
  free(sh->M);
  free(sh->MtM);
  free(sh->HR);
  free(sh);
}

/* dims: lmax, lmax_response, lmax_data, n, nr, ndw, nhr, niter */
void oracle_shared_dims(const oracle_shared *sh, int *dims) {
  dims[0] = sh->lmax;
  dims[1] = sh->lmax_response;
  dims[2] = sh->lmax_data;
  dims[3] = sh->n;
  dims[4] = sh->nr;
  dims[5] = sh->ndw;
  dims[6] = sh->nhr;
  dims[7] = sh->niter;
}
/* which: 0 rconv, 1 M, 2 MtM (lower, full n*n buffer), 3 HR_trans, 4 DW_dirs,
 *        5 scalars [threshold, norm_lambda, neg_lambda] */
void oracle_shared_copy(const oracle_shared *sh, int which, double *out) {
  size_t sz = 0;
  const double *src = NULL;
  switch (which) {
    case 0: src = sh->rconv; sz = (size_t)sh->nr * sh->ndw; break;
    case 1: src = sh->M; sz = (size_t)sh->ndw * sh->n; break;
    case 2: src = sh->MtM; sz = (size_t)sh->n * sh->n; break;
    case 3: src = sh->HR; sz = (size_t)sh->nhr * sh->n; break;
    case 4: src = sh->DW_dirs; sz = (size_t)sh->ndw * 2; break;
    case 5:
      out[0] = sh->threshold;
      out[1] = sh->norm_lambda;
      out[2] = sh->neg_lambda;
      return;
  }
  if (src) memcpy(out, src, sz * sizeof(double));
}
void oracle_shared_dwis(const oracle_shared *sh, int *out) {
  memcpy(out, sh->dwis, sizeof(int) * (size_t)sh->ndw);
}

/* ---- per-voxel CSD: CSD_Processor::operator() (dwi2fod.cpp:128-147) with
 *      load_data (:156-173), CSD::set (csd.h:237-243), iterate (:245-269) --- */
typedef struct {
  double *S, *F, *Mtb, *amps, *work, *HRT;
  int *neg, *old_neg;
} oracle_ws;

static void ws_alloc(const oracle_shared *sh, oracle_ws *w) {
  w->S = malloc(sizeof(double) * (size_t)sh->ndw);
  w->F = malloc(sizeof(double) * (size_t)sh->n);
  w->Mtb = malloc(sizeof(double) * (size_t)sh->n);
  w->amps = malloc(sizeof(double) * (size_t)sh->nhr);
  w->work = malloc(sizeof(double) * (size_t)sh->n * sh->n);
  w->HRT = malloc(sizeof(double) * (size_t)sh->nhr * sh->n);
  w->neg = malloc(sizeof(int) * (size_t)(sh->nhr + 1));
  w->old_neg = malloc(sizeof(int) * (size_t)(sh->nhr + 1));
}
static void ws_free(oracle_ws *w) {
  free(w->S); free(w->F); free(w->Mtb); free(w->amps); free(w->work); free(w->HRT);
  free(w->neg); free(w->old_neg);
}

/* status codes (shared with the product ABI): 0 masked out, 1 converged,
 * 2 hit niter, 3 non-finite input; 0x20 flag = Cholesky failed */
static int voxel_solve(const oracle_shared *sh, oracle_ws *w, const float *dwi, long vol_stride,
                       int masked_out, double *Fout, int *iters_out, uint32_t *negmask,
                       const uint32_t *warm) {
  const int n = sh->n, nr = sh->nr, ndw = sh->ndw, nhr = sh->nhr;
  const int nwords = (nhr + 31) / 32;
  if (negmask) memset(negmask, 0, sizeof(uint32_t) * (size_t)nwords);
  *iters_out = 0;
  int finite = 1;
  if (!masked_out) {
    for (int i = 0; i < ndw; i++) {
      double v = (double)dwi[(long)sh->dwis[i] * vol_stride];
      if (!isfinite(v)) {
        finite = 0;
        break;
      }
      w->S[i] = v < 0.0 ? 0.0 : v;
    }
  }
  if (masked_out || !finite) {
    for (int i = 0; i < n; i++) Fout[i] = 0.0;
    return masked_out ? 0 : 3;
  }
  /* csd.h:238-242 */
  for (int r = 0; r < n; r++) w->F[r] = 0.0;
  for (int r = 0; r < nr; r++) {
    double s = 0.0;
    for (int k = 0; k < ndw; k++) s += sh->rconv[r * ndw + k] * w->S[k];
    w->F[r] = s;
  }
  for (int c = 0; c < n; c++) {
    double s = 0.0;
    for (int k = 0; k < ndw; k++) s += sh->M[k * n + c] * w->S[k];
    w->Mtb[c] = s;
  }
  int nold = 1;
  w->old_neg[0] = -1;
  int status = 2, cholfail = 0, it;
  for (it = 0; it < sh->niter; it++) {
    int nneg = 0;
    if (it == 0 && warm) {
      /* warm start: the first negative set is supplied, not projected */
      for (int d = 0; d < nhr; d++)
        if ((warm[d >> 5] >> (d & 31)) & 1u) w->neg[nneg++] = d;
    } else {
      /* csd.h:246-250 */
      for (int d = 0; d < nhr; d++) {
        const double *h = sh->HR + (size_t)d * n;
        double s = 0.0;
        for (int i = 0; i < n; i++) s += h[i] * w->F[i];
        w->amps[d] = s;
        if (s < sh->threshold) w->neg[nneg++] = d;
      }
      /* csd.h:252-253: exact ordered index-list equality */
      if (nneg == nold && !memcmp(w->neg, w->old_neg, sizeof(int) * (size_t)nneg)) {
        status = 1;
        it++;
        break;
      }
    }
    /* csd.h:255-262: lower(work) = lower(Mt_M) + HR_T^T HR_T over the gathered rows */
    /* the product HR_T^T HR_T is formed first (row-outer so the inner loop
     * vectorises), then added to Mt_M, as Eigen evaluates `lower += A^T A` */
    double *P = w->HRT;
    for (int i = 0; i < n; i++)
      for (int j = 0; j <= i; j++) P[i * n + j] = 0.0;
    for (int q = 0; q < nneg; q++) {
      const double *h = sh->HR + (size_t)w->neg[q] * n;
      for (int i = 0; i < n; i++) {
        const double hi = h[i];
        double *Pi = P + (size_t)i * n;
        for (int j = 0; j <= i; j++) Pi[j] += hi * h[j];
      }
    }
    for (int i = 0; i < n; i++)
      for (int j = 0; j <= i; j++) w->work[i * n + j] = sh->MtM[i * n + j] + P[i * n + j];
    /* csd.h:264: F = LLT(work).solve(Mt_b) (info() is not checked upstream) */
    if (chol_lower(w->work, n)) cholfail = 1;
    for (int i = 0; i < n; i++) w->F[i] = w->Mtb[i];
    chol_solve(w->work, n, w->F);
    /* csd.h:266 */
    memcpy(w->old_neg, w->neg, sizeof(int) * (size_t)nneg);
    nold = nneg;
  }
  *iters_out = it;
  if (negmask && sh->niter > 0)
    for (int q = 0; q < nold; q++)
      if (w->old_neg[q] >= 0) negmask[w->old_neg[q] >> 5] |= 1u << (w->old_neg[q] & 31);
  for (int i = 0; i < n; i++) Fout[i] = w->F[i];
  return status | (cholfail ? 0x20 : 0);
}

/* ---- threaded driver: voxel rows handed out under a mutex, per-thread
 *      workspace copy (core/algo/threaded_loop.h:324-362) ------------------ */
typedef struct {
  const oracle_shared *sh;
  const float *dwi;
  long nvox, vox_stride, vol_stride, row;
  const uint8_t *mask;
  const uint32_t *warm;
  double *F;
  int *iters;
  uint32_t *negmask;
  uint8_t *status;
  long next;
  pthread_mutex_t mu;
} oracle_job;

static void *oracle_worker(void *arg) {
  oracle_job *j = (oracle_job *)arg;
  oracle_ws w;
  ws_alloc(j->sh, &w);
  const int nwords = (j->sh->nhr + 31) / 32;
  for (;;) {
    pthread_mutex_lock(&j->mu);
    long start = j->next;
    j->next += j->row;
    pthread_mutex_unlock(&j->mu);
    if (start >= j->nvox) break;
    long end = start + j->row < j->nvox ? start + j->row : j->nvox;
    for (long v = start; v < end; v++) {
      int it = 0;
      int st = voxel_solve(j->sh, &w, j->dwi + v * j->vox_stride, j->vol_stride,
                           j->mask ? !j->mask[v] : 0, j->F + v * j->sh->n, &it,
                           j->negmask ? j->negmask + v * nwords : NULL,
                           j->warm ? j->warm + v * nwords : NULL);
      if (j->iters) j->iters[v] = it;
      if (j->status) j->status[v] = (uint8_t)st;
    }
  }
  ws_free(&w);
  return NULL;
}

/* Solve nvox voxels.  dwi[v*vox_stride + vol*vol_stride] holds volume `vol`
 * of voxel v (float32, as read by dwi2fod).  Outputs FP64 F [nvox][n],
 * iterate() call counts, the final negative set as a bitmask [nvox][nwords]
 * and a status byte.  warm (nullable) supplies the first negative set. */
int oracle_solve(const oracle_shared *sh, const float *dwi, long nvox, long vox_stride,
                 long vol_stride, const uint8_t *mask, const uint32_t *warm, double *F,
                 int *iters, uint32_t *negmask, uint8_t *status, int nthreads) {
  oracle_job j;
  j.sh = sh;
  j.dwi = dwi;
  j.nvox = nvox;
  j.vox_stride = vox_stride;
  j.vol_stride = vol_stride;
  j.row = 64;
  j.mask = mask;
  j.warm = warm;
  j.F = F;
  j.iters = iters;
  j.negmask = negmask;
  j.status = status;
  j.next = 0;
  pthread_mutex_init(&j.mu, NULL);
  if (nthreads < 1) nthreads = 1;
  if (nthreads == 1) {
    oracle_worker(&j);
  } else {
    pthread_t *th = malloc(sizeof(pthread_t) * (size_t)nthreads);
    for (int t = 0; t < nthreads; t++) pthread_create(&th[t], NULL, oracle_worker, &j);
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    free(th);
  }
  pthread_mutex_destroy(&j.mu);
  return 0;
}
