// TEST INFRASTRUCTURE ONLY: FP64 C restatement of MRtrix3's FMLS FOD
// segmenter (src/dwi/fmls.cpp:159-311, FOD_lobe of src/dwi/fmls.h:60-160),
// threaded over voxels: the CPU baseline of fod2fixel and a second check of
// the GPU segmenter.  It keeps the reference's own data structure -- a vector
// of lobes with a mask over the directions each, lobes merged and erased by
// vector index, pending assignments re-indexed on every merge -- and
// get_peak's Newton search (core/math/SH.h:515-650) with the PrecomputedAL
// table (SH.h:435-460) and FastLookupSet::select_direction (set.cpp:340-354).
// The tables (directions, neighbours, weights, SH transform, Legendre table,
// grid) are passed in.  A voxel with a non-finite coefficient has no lobes.
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int ndir, lmax, nsh;
  const double *unit, *weight, *sh2amp, *al;
  const int *adj_off, *adj;
  int al_ndir, n_al;
  double al_inc;
  int num_az, num_el;
  double az_begin, el_begin, az_step, el_step;
  const int *grid_off, *grid;
  double integral_thr, peak_thr, merge_ratio;
} Seg;

typedef struct {
  unsigned char* mask;
  double max_peak, mean[3], integral;
  int neg, npeaks, cap;
  double* peaks;  // [cap][3]
} Lobe;

typedef struct {
  double* values;
  int* order;
  Lobe* lobes;  // ndir slots, buffers kept across voxels
  int* retro_dir;
  int* retro_lobe;
} Work;

static __thread const double* t_values;

static int cmp_order(const void* a, const void* b) {
  const int i = *(const int*)a, j = *(const int*)b;
  const double fi = fabs(t_values[i]), fj = fabs(t_values[j]);
  if (fi > fj) return -1;
  if (fi < fj) return 1;
  return i < j ? -1 : (i > j ? 1 : 0);
}

static void push_peak(Lobe* L, const double* p) {
  if (L->npeaks == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 4;
    L->peaks = realloc(L->peaks, sizeof(double) * 3 * L->cap);
  }
  memcpy(L->peaks + 3 * L->npeaks, p, sizeof(double) * 3);
  L->npeaks++;
}

static void lobe_init(const Seg* S, Lobe* L, int d, double v) {
  const double* u = S->unit + 3 * d;
  const double w = S->weight[d];
  memset(L->mask, 0, S->ndir);
  L->mask[d] = 1;
  L->max_peak = fabs(v);
  L->npeaks = 0;
  push_peak(L, u);
  for (int k = 0; k < 3; ++k) L->mean[k] = u[k] * fabs(v) * w;
  L->integral = fabs(v * w);
  L->neg = v <= 0.0;
}

static void lobe_add(const Seg* S, Lobe* L, int d, double v) {
  const double* u = S->unit + 3 * d;
  const double w = S->weight[d];
  L->mask[d] = 1;
  const double mult = (L->mean[0] * u[0] + L->mean[1] * u[1] + L->mean[2] * u[2]) > 0.0 ? 1.0 : -1.0;
  for (int k = 0; k < 3; ++k) L->mean[k] += u[k] * mult * fabs(v) * w;
  L->integral += fabs(v * w);
}

static void lobe_merge(const Seg* S, Lobe* A, const Lobe* B) {
  for (int i = 0; i < S->ndir; ++i) A->mask[i] |= B->mask[i];
  if (B->max_peak > A->max_peak) {
    A->max_peak = B->max_peak;
    // B's peaks in front of A's
    double* old = malloc(sizeof(double) * 3 * (A->npeaks ? A->npeaks : 1));
    const int n_old = A->npeaks;
    memcpy(old, A->peaks, sizeof(double) * 3 * n_old);
    A->npeaks = 0;
    for (int i = 0; i < B->npeaks; ++i) push_peak(A, B->peaks + 3 * i);
    for (int i = 0; i < n_old; ++i) push_peak(A, old + 3 * i);
    free(old);
  } else {
    for (int i = 0; i < B->npeaks; ++i) push_peak(A, B->peaks + 3 * i);
  }
  const double mult = (A->mean[0] * B->mean[0] + A->mean[1] * B->mean[1] + A->mean[2] * B->mean[2]) > 0.0 ? 1.0 : -1.0;
  for (int k = 0; k < 3; ++k) A->mean[k] += B->mean[k] * B->integral * mult;
  A->integral += B->integral;
}

static int is_adjacent(const Seg* S, const Lobe* L, int d) {
  for (int e = S->adj_off[d]; e < S->adj_off[d + 1]; ++e)
    if (L->mask[S->adj[e]]) return 1;
  return 0;
}

static void derivatives(const Seg* S, const double* sh, double el, double az, double* o) {
  const double sel = sin(el);
  const int atpole = sel < 1e-4;
  double f2 = el / S->al_inc, f1;
  int i = (int)f2;
  if (i < 0) {
    i = 0; f1 = 1.0; f2 = 0.0;
  } else if (i >= S->al_ndir - 1) {
    i = S->al_ndir - 1; f1 = 1.0; f2 = 0.0;
  } else {
    f2 -= i; f1 = 1.0 - f2;
  }
  const double* p1 = S->al + (size_t)i * S->n_al;
  const double* p2 = p1 + S->n_al;
#define AL(l, m) (f2 != 0.0 ? f1 * p1[(l) * (l) / 4 + (m)] + f2 * p2[(l) * (l) / 4 + (m)] : f1 * p1[(l) * (l) / 4 + (m)])
#define IX(l, m) ((l) * ((l) + 1) / 2 + (m))
  double amp = sh[0] * AL(0, 0), d_el = 0, d_az = 0, d2_el = 0, d2_elaz = 0, d2_az = 0;
  for (int l = 2; l <= S->lmax; l += 2) {
    const double v = sh[IX(l, 0)];
    amp += v * AL(l, 0);
    d_el += v * sqrt((double)(l * (l + 1))) * AL(l, 1);
    d2_el += v * (sqrt((double)(l * (l + 1) * (l - 1) * (l + 2))) * AL(l, 2) - l * (l + 1) * AL(l, 0)) / 2.0;
  }
  for (int m = 1; m <= S->lmax; ++m) {
    const double caz = sqrt(2.0) * cos(m * az), saz = sqrt(2.0) * sin(m * az);
    for (int l = (m & 1) ? m + 1 : m; l <= S->lmax; l += 2) {
      const double vp = sh[IX(l, m)], vm = sh[IX(l, -m)];
      amp += (vp * caz + vm * saz) * AL(l, m);
      double tmp = sqrt((double)((l + m) * (l - m + 1))) * AL(l, m - 1);
      if (l > m) tmp -= sqrt((double)((l - m) * (l + m + 1))) * AL(l, m + 1);
      tmp /= -2.0;
      d_el += (vp * caz + vm * saz) * tmp;
      double tmp2 = -((l + m) * (l - m + 1) + (l - m) * (l + m + 1)) * AL(l, m);
      if (m == 1)
        tmp2 -= sqrt((double)((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2))) * AL(l, 1);
      else
        tmp2 += sqrt((double)((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2))) * AL(l, m - 2);
      if (l > m + 1) tmp2 += sqrt((double)((l - m) * (l + m + 1) * (l - m - 1) * (l + m + 2))) * AL(l, m + 2);
      tmp2 /= 4.0;
      d2_el += (vp * caz + vm * saz) * tmp2;
      if (atpole) {
        d_az += (vm * caz - vp * saz) * tmp;
      } else {
        d_az += m * (vm * caz - vp * saz) * AL(l, m);
        d2_elaz += m * (vm * caz - vp * saz) * tmp;
        d2_az -= (vp * caz + vm * saz) * m * m * AL(l, m);
      }
    }
  }
#undef AL
#undef IX
  if (!atpole) {
    d_az /= sel;
    d2_elaz /= sel;
    d2_az /= sel * sel;
  }
  o[0] = amp; o[1] = d_el; o[2] = d_az; o[3] = d2_el; o[4] = d2_elaz; o[5] = d2_az;
}

static double get_peak(const Seg* S, const double* sh, double* u) {
  for (int it = 0; it < 50; ++it) {
    const double az = atan2(u[1], u[0]), el = atan2(hypot(u[0], u[1]), u[2]);
    double dv[6];
    derivatives(S, sh, el, az, dv);
    double del = sqrt(dv[1] * dv[1] + dv[2] * dv[2]), daz = 0.0;
    if (del != 0.0) {
      daz = dv[2] / del;
      del = dv[1] / del;
    }
    const double dSH_dt = daz * dv[2] + del * dv[1];
    const double d2SH_dt2 = daz * daz * dv[5] + 2.0 * daz * del * dv[4] + del * del * dv[3];
    double dt = d2SH_dt2 != 0.0 ? (-dSH_dt / d2SH_dt2) : 0.2;
    if (dt < 0.0) dt = -dt;
    if (dt > 0.2) dt = 0.2;
    del *= dt;
    daz *= dt;
    u[0] += del * cos(az) * cos(el) - daz * sin(az);
    u[1] += del * sin(az) * cos(el) + daz * cos(az);
    u[2] -= del * sin(el);
    const double n = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    u[0] /= n; u[1] /= n; u[2] /= n;
    if (dt < 1e-4) return dv[0];
  }
  u[0] = u[1] = u[2] = NAN;
  return NAN;
}

static int select_direction(const Seg* S, const double* p) {
  const double az = atan2(p[1], p[0]), el = acos(p[2] > 1.0 ? 1.0 : (p[2] < -1.0 ? -1.0 : p[2]));
  long ai = (long)floor((az - S->az_begin) / S->az_step), ei = (long)floor((el - S->el_begin) / S->el_step);
  if (ai < 0) ai = 0;
  if (ai >= S->num_az) ai = S->num_az - 1;
  if (ei < 0) ei = 0;
  if (ei >= S->num_el) ei = S->num_el - 1;
  const long c = ai * S->num_el + ei;
  int best = S->grid[S->grid_off[c]];
  double best_dp = fabs(p[0] * S->unit[3 * best] + p[1] * S->unit[3 * best + 1] + p[2] * S->unit[3 * best + 2]);
  for (int e = S->grid_off[c] + 1; e < S->grid_off[c + 1]; ++e) {
    const int d = S->grid[e];
    const double dp = fabs(p[0] * S->unit[3 * d] + p[1] * S->unit[3 * d + 1] + p[2] * S->unit[3 * d + 2]);
    if (dp > best_dp) {
      best_dp = dp;
      best = d;
    }
  }
  return best;
}

static void erase_lobe(Lobe* lobes, int n, int j) {
  Lobe keep = lobes[j];  // its buffers go to the end of the pool
  memmove(lobes + j, lobes + j + 1, sizeof(Lobe) * (n - j - 1));
  lobes[n - 1] = keep;
}

static int segment_voxel(const Seg* S, Work* w, const double* sh, float* out, int max_out) {
  const int nd = S->ndir;
  if (!(sh[0] > 0.0) || !isfinite(sh[0])) return 0;
  for (int k = 1; k < S->nsh; ++k)
    if (!isfinite(sh[k])) return 0;
  for (int d = 0; d < nd; ++d) {
    double s = 0.0;
    for (int k = 0; k < S->nsh; ++k) s += S->sh2amp[(size_t)d * S->nsh + k] * sh[k];
    w->values[d] = s;
    w->order[d] = d;
  }
  t_values = w->values;
  qsort(w->order, nd, sizeof(int), cmp_order);
  if (w->values[w->order[0]] <= 0.0) return 0;
  int nl = 0, nr = 0;
  int adj[64];
  for (int k = 0; k < nd; ++k) {
    const int d = w->order[k];
    const double v = w->values[d];
    int na = 0;
    for (int l = 0; l < nl && na < 64; ++l)
      if ((v <= 0.0) == w->lobes[l].neg && is_adjacent(S, &w->lobes[l], d)) adj[na++] = l;
    if (na == 0) {
      lobe_init(S, &w->lobes[nl++], d, v);
    } else if (na == 1) {
      lobe_add(S, &w->lobes[adj[0]], d, v);
    } else if (fabs(v) / w->lobes[adj[na - 1]].max_peak > S->merge_ratio) {
      for (int j = 1; j < na; ++j) lobe_merge(S, &w->lobes[adj[0]], &w->lobes[adj[j]]);
      lobe_add(S, &w->lobes[adj[0]], d, v);
      for (int r = 0; r < nr; ++r) {
        int modified = 0;
        for (int j = 1; j < na; ++j)
          if (w->retro_lobe[r] == adj[j]) {
            w->retro_lobe[r] = adj[0];
            modified = 1;
          }
        if (!modified) {
          int idx = w->retro_lobe[r];
          for (int j = na - 1; j >= 1; --j)
            if (adj[j] < idx) --idx;
          w->retro_lobe[r] = idx;
        }
      }
      for (int j = na - 1; j >= 1; --j) erase_lobe(w->lobes, nl--, adj[j]);
    } else {
      w->retro_dir[nr] = d;
      w->retro_lobe[nr] = adj[0];
      ++nr;
    }
  }
  for (int r = 0; r < nr; ++r) lobe_add(S, &w->lobes[w->retro_lobe[r]], w->retro_dir[r], w->values[w->retro_dir[r]]);
  int nout = 0;
  for (int l = 0; l < nl; ++l) {
    Lobe* L = &w->lobes[l];
    if (L->neg || L->integral < S->integral_thr) continue;
    for (int pi = 0; pi < L->npeaks; ++pi) {
      double u[3] = {L->peaks[3 * pi], L->peaks[3 * pi + 1], L->peaks[3 * pi + 2]};
      const double val = get_peak(S, sh, u);
      if (!(isfinite(val) && isfinite(u[0]) && isfinite(u[1]) && isfinite(u[2]))) continue;
      double max_dp = 0.0;
      int nearest = L->npeaks;
      for (int j = 0; j < L->npeaks; ++j) {
        const double dp = fabs(u[0] * L->peaks[3 * j] + u[1] * L->peaks[3 * j + 1] + u[2] * L->peaks[3 * j + 2]);
        if (dp > max_dp) {
          max_dp = dp;
          nearest = j;
        }
      }
      if (nearest != pi) continue;
      if (!L->mask[select_direction(S, u)]) continue;
      memcpy(L->peaks + 3 * pi, u, sizeof(u));
      if (pi == 0) L->max_peak = val;
    }
    if (L->max_peak < S->peak_thr) continue;
    if (nout < max_out) {
      const double n2 = L->mean[0] * L->mean[0] + L->mean[1] * L->mean[1] + L->mean[2] * L->mean[2];
      const double n = n2 > 0.0 ? sqrt(n2) : 1.0;
      float* f = out + (size_t)nout * 8;
      for (int k = 0; k < 3; ++k) {
        f[k] = (float)(n2 > 0.0 ? L->mean[k] / n : L->mean[k]);
        f[3 + k] = (float)L->peaks[k];
      }
      f[6] = (float)L->integral;
      f[7] = (float)L->max_peak;
    }
    ++nout;
  }
  return nout;
}

typedef struct {
  const Seg* S;
  const double* sh;
  int max_out;
  int* counts;
  float* fixels;
  long begin, end;
} Task;

static void* run_task(void* arg) {
  Task* t = (Task*)arg;
  const Seg* S = t->S;
  const int nd = S->ndir;
  Work w;
  w.values = malloc(sizeof(double) * nd);
  w.order = malloc(sizeof(int) * nd);
  w.retro_dir = malloc(sizeof(int) * nd);
  w.retro_lobe = malloc(sizeof(int) * nd);
  w.lobes = calloc(nd, sizeof(Lobe));
  for (int i = 0; i < nd; ++i) w.lobes[i].mask = malloc(nd);
  for (long v = t->begin; v < t->end; ++v)
    t->counts[v] = segment_voxel(S, &w, t->sh + (size_t)v * S->nsh, t->fixels + (size_t)v * t->max_out * 8,
                                 t->max_out);
  for (int i = 0; i < nd; ++i) {
    free(w.lobes[i].mask);
    free(w.lobes[i].peaks);
  }
  free(w.lobes);
  free(w.values);
  free(w.order);
  free(w.retro_dir);
  free(w.retro_lobe);
  return NULL;
}

// counts [n], fixels [n][max_out][8] (mean dir, peak dir, integral, max peak)
// for the SH rows sh [n][nsh].
int oracle_fmls_segment(int ndir, int lmax, int nsh, const double* unit, const double* weight, const int* adj_off,
                        const int* adj, const double* sh2amp, int al_ndir, int n_al, double al_inc, const double* al,
                        int num_az, int num_el, double az_begin, double el_begin, double az_step, double el_step,
                        const int* grid_off, const int* grid, double integral_thr, double peak_thr,
                        double merge_ratio, const double* sh, long n, int max_out, int* counts, float* fixels,
                        int nthreads) {
  Seg S = {ndir, lmax, nsh, unit, weight, sh2amp, al, adj_off, adj, al_ndir, n_al, al_inc, num_az, num_el, az_begin,
           el_begin, az_step, el_step, grid_off, grid, integral_thr, peak_thr, merge_ratio};
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  Task task[256];
  const long chunk = (n + nthreads - 1) / nthreads;
  int started = 0;
  for (int i = 0; i < nthreads; ++i) {
    task[i] = (Task){&S, sh, max_out, counts, fixels, i * chunk, (i + 1) * chunk < n ? (i + 1) * chunk : n};
    if (task[i].begin >= task[i].end) break;
    if (pthread_create(&th[i], NULL, run_task, &task[i]) != 0) return -1;
    ++started;
  }
  for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
  return 0;
}
