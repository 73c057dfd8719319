// TEST INFRASTRUCTURE ONLY: FP64 C restatement of MRtrix3's ICLS solver
// (core/math/constrained_least_squares.h:241-370, ICLS::Solver::operator()),
// the CPU baseline of the GPU multi-tissue CSD and a second checker beside
// oracle/icls_ref.py (which it is tested against).  As the reference, it
// forms B_a B_a^T over the active constraints in index order and refactors it
// (Cholesky) for every solve.  The problem tables come from the Python
// restatement of ICLS::Problem (b2d, normalised B, t, L).  Voxels are split
// over POSIX threads.
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int nmeas, nparam, ncons, num_eq, max_niter;
  double reg, tol;
  const double* b2d;  // [nmeas][nparam]
  const double* B;    // [ncons][nparam]
  const double* t;    // [ncons] or NULL
  const double* L;    // [nparam][nparam] lower, row-major
} Problem;

typedef struct {
  double *yu, *cu, *c, *lam, *lp, *l, *S, *x;
  int *active, *idx;
} Work;

static int solve_one(const Problem* P, Work* w, const double* b, double* xout) {
  const int N = P->nparam, M = P->ncons, num_ineq = M - P->num_eq;
  for (int j = 0; j < N; ++j) {
    double s = 0.0;
    for (int i = 0; i < P->nmeas; ++i) s += P->b2d[(size_t)i * N + j] * b[i];
    w->yu[j] = s;
  }
  for (int m = 0; m < M; ++m) {
    double s = 0.0;
    for (int j = 0; j < N; ++j) s += P->B[(size_t)m * N + j] * w->yu[j];
    if (P->t) s -= P->t[m];
    w->cu[m] = s;
    w->c[m] = s;
    w->lam[m] = w->lp[m] = 0.0;
    w->active[m] = m >= num_ineq;
  }
  memcpy(w->x, w->yu, sizeof(double) * N);
  int niter = 0;
  while (num_ineq > 0) {
    int imin = 0;
    for (int m = 1; m < num_ineq; ++m)
      if (w->c[m] < w->c[imin]) imin = m;
    if (!(w->c[imin] < -P->tol)) break;
    int changed = !w->active[imin];
    w->active[imin] = 1;
    for (;;) {
      int na = 0;
      for (int m = 0; m < M; ++m)
        if (w->active[m]) {
          w->idx[na] = m;
          w->l[na] = -w->cu[m];
          ++na;
        }
      // S = B_a B_a^T + reg I (lower), Cholesky in place
      for (int i = 0; i < na; ++i) {
        const double* bi = P->B + (size_t)w->idx[i] * N;
        for (int j = 0; j <= i; ++j) {
          const double* bj = P->B + (size_t)w->idx[j] * N;
          double s = 0.0;
          for (int k = 0; k < N; ++k) s += bi[k] * bj[k];
          w->S[(size_t)i * na + j] = s + (i == j ? P->reg : 0.0);
        }
      }
      for (int j = 0; j < na; ++j) {
        double d = w->S[(size_t)j * na + j];
        for (int k = 0; k < j; ++k) d -= w->S[(size_t)j * na + k] * w->S[(size_t)j * na + k];
        d = sqrt(d);
        w->S[(size_t)j * na + j] = d;
        for (int i = j + 1; i < na; ++i) {
          double s = w->S[(size_t)i * na + j];
          for (int k = 0; k < j; ++k) s -= w->S[(size_t)i * na + k] * w->S[(size_t)j * na + k];
          w->S[(size_t)i * na + j] = s / d;
        }
      }
      for (int i = 0; i < na; ++i) {
        double s = w->l[i];
        for (int k = 0; k < i; ++k) s -= w->S[(size_t)i * na + k] * w->l[k];
        w->l[i] = s / w->S[(size_t)i * na + i];
      }
      for (int i = na - 1; i >= 0; --i) {
        double s = w->l[i];
        for (int k = i + 1; k < na; ++k) s -= w->S[(size_t)k * na + i] * w->l[k];
        w->l[i] = s / w->S[(size_t)i * na + i];
      }
      double smin = INFINITY;
      int sidx = 0, a = 0;
      for (int n = 0; n < num_ineq; ++n) {
        if (w->active[n]) {
          if (w->l[a] < 0.0) {
            const double s = w->lp[n] / (w->lp[n] - w->l[a]);
            if (s < smin) {
              smin = s;
              sidx = n;
            }
          }
          w->lam[n] = w->l[a];
          ++a;
        } else {
          w->lam[n] = 0.0;
        }
      }
      if (!isfinite(smin)) {
        for (int j = 0; j < N; ++j) {
          double s = w->yu[j];
          for (int p = 0; p < na; ++p) s += P->B[(size_t)w->idx[p] * N + j] * w->l[p];
          w->x[j] = s;
        }
        break;
      }
      if (w->active[sidx]) changed = 1;
      w->active[sidx] = 0;
    }
    memcpy(w->lp, w->lam, sizeof(double) * M);
    ++niter;
    if (!changed || niter > P->max_niter) break;
    for (int m = 0; m < M; ++m) {
      double s = 0.0;
      for (int j = 0; j < N; ++j) s += P->B[(size_t)m * N + j] * w->x[j];
      if (P->t) s -= P->t[m];
      w->c[m] = s;
    }
  }
  for (int i = N - 1; i >= 0; --i) {  // L^T x = y
    double s = w->x[i];
    for (int k = i + 1; k < N; ++k) s -= P->L[(size_t)k * N + i] * w->x[k];
    w->x[i] = s / P->L[(size_t)i * N + i];
  }
  memcpy(xout, w->x, sizeof(double) * N);
  return niter;
}

typedef struct {
  const Problem* P;
  const double* b;
  double* x;
  int* niter;
  long begin, end;
} Task;

static void* run_task(void* arg) {
  Task* t = (Task*)arg;
  const Problem* P = t->P;
  const int M = P->ncons, N = P->nparam;
  Work w;
  w.yu = malloc(sizeof(double) * N);
  w.x = malloc(sizeof(double) * N);
  w.cu = malloc(sizeof(double) * M);
  w.c = malloc(sizeof(double) * M);
  w.lam = malloc(sizeof(double) * M);
  w.lp = malloc(sizeof(double) * M);
  w.l = malloc(sizeof(double) * M);
  w.S = malloc(sizeof(double) * (size_t)M * M);
  w.active = malloc(sizeof(int) * M);
  w.idx = malloc(sizeof(int) * M);
  for (long v = t->begin; v < t->end; ++v)
    t->niter[v] = solve_one(P, &w, t->b + (size_t)v * P->nmeas, t->x + (size_t)v * N);
  free(w.yu);
  free(w.x);
  free(w.cu);
  free(w.c);
  free(w.lam);
  free(w.lp);
  free(w.l);
  free(w.S);
  free(w.active);
  free(w.idx);
  return NULL;
}

// x [n][nparam], niter [n]: the solver for each row of b [n][nmeas].
int oracle_icls_solve(int nmeas, int nparam, int ncons, int num_eq, int max_niter, double reg, double tol,
                      const double* b2d, const double* B, const double* t, const double* L, const double* b, long n,
                      double* x, int* niter, int nthreads) {
  Problem P = {nmeas, nparam, ncons, num_eq, max_niter, reg, tol, b2d, B, t, L};
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  Task task[256];
  const long chunk = (n + nthreads - 1) / nthreads;
  int started = 0;
  for (int i = 0; i < nthreads; ++i) {
    task[i] = (Task){&P, b, x, niter, i * chunk, (i + 1) * chunk < n ? (i + 1) * chunk : n};
    if (task[i].begin >= task[i].end) break;
    if (pthread_create(&th[i], NULL, run_task, &task[i]) != 0) return -1;
    ++started;
  }
  for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
  return 0;
}
