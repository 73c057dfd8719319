// FMLS FOD segmentation of one voxel (MRtrix3 src/dwi/fmls.cpp:159-311,
// src/dwi/fmls.h:60-160), written once for the GPU kernel (fmls.cu) and for
// a host build that the CPU tests compare with the restatement in the oracle.
//
// The reference keeps a vector of lobes, each with a mask over the 1281
// directions, erases merged lobes from the vector and re-indexes the pending
// "retrospective" assignments on every merge.  Here a lobe is named by the
// order it was created in: a direction's label is the lobe that took it, a
// merged lobe points at the lobe it merged into (parent), and a lobe's
// current identity is the end of that chain.  The survivor of a merge is
// the adjacent lobe created first, which is the first of them in the
// reference's vector, so creation order among surviving lobes is the
// vector's order, a pending assignment follows its lobe through merges as
// the re-indexing there does, and a lobe's mask is every direction whose
// label leads to it.  A lobe's peak directions are a linked list (a merge
// puts the other lobe's peaks in front when its peak is larger, else
// behind).  Every array of the workspace holds one entry per direction.
#pragma once

#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define FMLS_HD __host__ __device__
#else
#define FMLS_HD
#endif

namespace fmls {

constexpr int kMaxAdj = 16;      // neighbours a direction may have
constexpr double kMaxDirChange = 0.2;    // SH.h: MAX_DIR_CHANGE
constexpr double kAngleTolerance = 1e-4; // SH.h: ANGLE_TOLERANCE

FMLS_HD inline bool finite(double x) {
#ifdef __CUDA_ARCH__
  return isfinite(x);
#else
  return std::isfinite(x);
#endif
}

struct Tables {
  int ndir, lmax, nsh;
  const double* unit;     // [ndir][3]
  const double* weight;   // [ndir] integration weights
  const int* adj_off;     // [ndir + 1]
  const int* adj;         // neighbour lists
  const double* sh2amp;   // [ndir][nsh]
  int al_ndir, n_al;      // PrecomputedAL: elevations, entries per row
  double al_inc;
  const double* al;       // [al_ndir][n_al]
  int num_az, num_el;     // FastLookupSet grid
  double az_begin, el_begin, az_step, el_step;
  const int* grid_off;    // [num_az * num_el + 1]
  const int* grid;
  double integral_threshold, peak_value_threshold, merge_ratio;
  // optional: the square roots derivatives() takes of integer products, per
  // (l, m) four of them (dsqrt_index); NULL computes them on the spot (the
  // values are the same: a correctly rounded square root of an exact integer)
  const double* dsqrt = nullptr;
  // optional: sh2amp transposed, [nsh][ndir] (the device reads it coalesced)
  const double* sh2amp_t = nullptr;
};

// Slots of Tables::dsqrt for degree l, order m (0 <= m <= l <= lmax):
// [0] sqrt((l+m)(l-m+1)), [1] sqrt((l-m)(l+m+1)),
// [2] sqrt((l+m)(l-m+1)(l+m-1)(l-m+2)), [3] sqrt((l-m)(l+m+1)(l-m-1)(l+m+2)).
FMLS_HD inline int dsqrt_index(int l, int m) { return 4 * (l * (l + 1) / 2 + m); }
FMLS_HD inline double dsqrt_value(int l, int m, int which) {
  double x;
  switch (which) {
    case 0: x = (double)((l + m) * (l - m + 1)); break;
    case 1: x = (double)((l - m) * (l + m + 1)); break;
    case 2: x = (double)((l + m) * (l - m + 1) * (l + m - 1) * (l - m + 2)); break;
    default: x = (double)((l - m) * (l + m + 1) * (l - m - 1) * (l + m + 2)); break;
  }
  return x > 0.0 ? sqrt(x) : 0.0;
}

// One voxel in flight.  values, order and label have one entry per
// direction, the lobe arrays one per lobe (at most one per direction), the
// pending lists one per direction.  I is the type of the labels and lobe
// links (a signed type that holds -1 and every lobe index), O that of the
// order entries.
template <class I, class O>
struct WorkT {
  double* values;
  O* order;
  I* label;
  I* parent;
  I* neg;
  double* max_peak;
  double* mean;       // [3 lobes]
  double* integral;
  I* peak_head;
  I* peak_tail;
  I* peak_next;
  double* peak_dir;   // [3 lobes]; peak p was created with lobe p
  int* retro_dir;
  int* retro_lobe;
};
using Work = WorkT<int, int>;

struct Fixel {  // fod2fixel's per-fixel values
  float mean_dir[3], peak_dir[3], integral, max_peak;
};

FMLS_HD inline bool before(const double* v, int ndir, int a, int b) {
  // the multimap order of fmls.cpp:172-176: |value| descending, then index
  if (a >= ndir) return false;
  if (b >= ndir) return true;
  const double fa = fabs(v[a]), fb = fabs(v[b]);
  return fa > fb || (fa == fb && a < b);
}

template <class W>
FMLS_HD inline int root(const W& w, int l) {
  while (w.parent[l] != l) l = w.parent[l];
  return l;
}

template <class W>
FMLS_HD inline void lobe_add(const Tables& t, const W& w, int r, int d, double value) {
  // FOD_lobe::add (fmls.h:82-91)
  const double* u = t.unit + 3 * d;
  double* m = w.mean + 3 * r;
  w.label[d] = r;
  const double mult = (m[0] * u[0] + m[1] * u[1] + m[2] * u[2]) > 0.0 ? 1.0 : -1.0;
  const double av = fabs(value), wt = t.weight[d];
  for (int k = 0; k < 3; ++k) m[k] += u[k] * mult * av * wt;
  w.integral[r] += fabs(value * wt);
}

template <class W>
FMLS_HD inline void lobe_merge(const W& w, int a, int b) {
  // FOD_lobe::merge (fmls.h:111-126): b into a
  if (w.max_peak[b] > w.max_peak[a]) {
    w.max_peak[a] = w.max_peak[b];
    w.peak_next[w.peak_tail[b]] = w.peak_head[a];
    w.peak_head[a] = w.peak_head[b];
  } else {
    w.peak_next[w.peak_tail[a]] = w.peak_head[b];
    w.peak_tail[a] = w.peak_tail[b];
  }
  double* ma = w.mean + 3 * a;
  const double* mb = w.mean + 3 * b;
  const double mult = (ma[0] * mb[0] + ma[1] * mb[1] + ma[2] * mb[2]) > 0.0 ? 1.0 : -1.0;
  const double ib = w.integral[b];
  for (int k = 0; k < 3; ++k) ma[k] += mb[k] * ib * mult;
  w.integral[a] += ib;
  w.parent[b] = a;
}

// The region growing of fmls.cpp:178-246 over the directions in w.order.
// Returns the number of lobes created; *n_retro the pending assignments.
// max_lobes bounds the lobe arrays of w: a voxel that would create more
// returns -1 (the caller repeats it with larger arrays).
template <class W>
FMLS_HD inline int grow(const Tables& t, const W& w, int* n_retro, int max_lobes = 1 << 30) {
  int nl = 0, nr = 0;
  for (int d = 0; d < t.ndir; ++d) w.label[d] = -1;
  for (int k = 0; k < t.ndir; ++k) {
    const int d = w.order[k];
    const double v = w.values[d];
    const int vneg = v <= 0.0 ? 1 : 0;
    int adj[kMaxAdj];
    int na = 0;
    for (int e = t.adj_off[d]; e < t.adj_off[d + 1]; ++e) {
      const int lab = w.label[t.adj[e]];
      if (lab < 0) continue;
      const int r = root(w, lab);
      if (w.neg[r] != vneg) continue;
      int pos = na;
      bool dup = false;
      for (int q = 0; q < na; ++q) {
        if (adj[q] == r) { dup = true; break; }
        if (adj[q] > r && pos == na) pos = q;
      }
      if (dup || na == kMaxAdj) continue;
      for (int q = na; q > pos; --q) adj[q] = adj[q - 1];
      adj[pos] = r;
      ++na;
    }
    if (na == 0) {
      // FOD_lobe constructor (fmls.h:60-72)
      if (nl >= max_lobes) return -1;
      const double* u = t.unit + 3 * d;
      const double av = fabs(v), wt = t.weight[d];
      w.parent[nl] = nl;
      w.neg[nl] = vneg;
      w.max_peak[nl] = av;
      w.peak_head[nl] = w.peak_tail[nl] = nl;
      w.peak_next[nl] = -1;
      for (int q = 0; q < 3; ++q) {
        w.peak_dir[3 * nl + q] = u[q];
        w.mean[3 * nl + q] = u[q] * av * wt;
      }
      w.integral[nl] = fabs(v * wt);
      w.label[d] = nl;
      ++nl;
    } else if (na == 1) {
      lobe_add(t, w, adj[0], d, v);
    } else if (fabs(v) / w.max_peak[adj[na - 1]] > t.merge_ratio) {
      for (int q = 1; q < na; ++q) lobe_merge(w, adj[0], adj[q]);
      lobe_add(t, w, adj[0], d, v);
    } else {
      w.retro_dir[nr] = d;
      w.retro_lobe[nr] = adj[0];
      ++nr;
    }
  }
  *n_retro = nr;
  return nl;
}

// PrecomputedAL::set (SH.h:435-460): the table row at or below elevation
// el and the weights of it and of the next row.
FMLS_HD inline void al_weights(const Tables& t, double el, int* row, double* w1, double* w2) {
  double f2 = el / t.al_inc, f1;
  int i = (int)f2;
  if (i < 0) {
    i = 0; f1 = 1.0; f2 = 0.0;
  } else if (i >= t.al_ndir - 1) {
    i = t.al_ndir - 1; f1 = 1.0; f2 = 0.0;
  } else {
    f2 -= i; f1 = 1.0 - f2;
  }
  *row = i;
  *w1 = f1;
  *w2 = f2;
}

// PrecomputedAL::get: entry k (= l^2/4 + m) interpolated between the rows
// (the next row is read only with a non-zero weight).
FMLS_HD inline double al_value(const Tables& t, int row, double f1, double f2, int k) {
  const double* p1 = t.al + (long long)row * t.n_al;
  double v = f1 * p1[k];
  if (f2 != 0.0) v += f2 * p1[t.n_al + k];
  return v;
}

// SH::derivatives (SH.h:569-650) given the interpolated Legendre values as
// AL(l, m).  SH is anything that gives coefficient i as sh[i] (a double
// pointer, or a view of FP32 coefficients, which convert to double exactly).
template <class SH, class ALF>
FMLS_HD inline void derivatives_with(const Tables& t, const SH& sh, const ALF& AL, double el, double az,
                                     double* out6) {
  const double sel = sin(el);
  const bool atpole = sel < 1e-4;
  auto IDX = [](int l, int m) { return l * (l + 1) / 2 + m; };
  const int lmax = t.lmax;
  auto SQ = [&](int l, int m, int which) {
    return t.dsqrt ? t.dsqrt[dsqrt_index(l, m) + which] : dsqrt_value(l, m, which);
  };
  double amp = sh[0] * AL(0, 0);
  double d_el = 0.0, d_az = 0.0, d2_el = 0.0, d2_elaz = 0.0, d2_az = 0.0;
  for (int l = 2; l <= lmax; l += 2) {
    const double v = sh[IDX(l, 0)];
    amp += v * AL(l, 0);
    d_el += v * SQ(l, 0, 1) * AL(l, 1);                                        // sqrt(l (l+1))
    d2_el += v * (SQ(l, 0, 3) * AL(l, 2) - l * (l + 1) * AL(l, 0)) / 2.0;    // sqrt(l (l+1) (l-1) (l+2))
  }
  const double sqrt2 = 1.4142135623730951;
  for (int m = 1; m <= lmax; ++m) {
    double sm, cm;
#ifdef __CUDA_ARCH__
    sincos(m * az, &sm, &cm);
#else
    sm = sin(m * az);
    cm = cos(m * az);
#endif
    const double caz = sqrt2 * cm, saz = sqrt2 * sm;
    for (int l = (m & 1) ? m + 1 : m; l <= lmax; l += 2) {
      const double vp = sh[IDX(l, m)], vm = sh[IDX(l, -m)];
      amp += (vp * caz + vm * saz) * AL(l, m);
      double tmp = SQ(l, m, 0) * AL(l, m - 1);
      if (l > m) tmp -= SQ(l, m, 1) * AL(l, m + 1);
      tmp /= -2.0;
      d_el += (vp * caz + vm * saz) * tmp;
      double tmp2 = -((l + m) * (l - m + 1) + (l - m) * (l + m + 1)) * AL(l, m);
      if (m == 1)
        tmp2 -= SQ(l, m, 2) * AL(l, 1);
      else
        tmp2 += SQ(l, m, 2) * AL(l, m - 2);
      if (l > m + 1) tmp2 += SQ(l, m, 3) * AL(l, m + 2);
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
  if (!atpole) {
    d_az /= sel;
    d2_elaz /= sel;
    d2_az /= sel * sel;
  }
  out6[0] = amp; out6[1] = d_el; out6[2] = d_az; out6[3] = d2_el; out6[4] = d2_elaz; out6[5] = d2_az;
}

// SH::derivatives with the precomputed Legendre table (SH.h:569-650).
template <class SH>
FMLS_HD inline void derivatives(const Tables& t, const SH& sh, double el, double az, double* out6) {
  int row;
  double f1, f2;
  al_weights(t, el, &row, &f1, &f2);
  auto AL = [&](int l, int m) { return al_value(t, row, f1, f2, l * l / 4 + m); };
  derivatives_with(t, sh, AL, el, az, out6);
}

// One Newton step of SH::get_peak (SH.h:515-560) from u (updated in
// place).  Returns true when the step was below the angle tolerance: the
// peak has converged and *val is the amplitude there.
// DER(el, az, dv) evaluates the six derivatives there.
template <class DER>
FMLS_HD inline bool newton_step(const DER& der, double* u, double* val) {
  const double az = atan2(u[1], u[0]);
  const double el = atan2(hypot(u[0], u[1]), u[2]);
  double dv[6];
  der(el, az, dv);
  double del = sqrt(dv[1] * dv[1] + dv[2] * dv[2]);
  double daz = 0.0;
  if (del != 0.0) {
    daz = dv[2] / del;
    del = dv[1] / del;
  }
  const double dSH_dt = daz * dv[2] + del * dv[1];
  const double d2SH_dt2 = daz * daz * dv[5] + 2.0 * daz * del * dv[4] + del * del * dv[3];
  double dt = d2SH_dt2 != 0.0 ? (-dSH_dt / d2SH_dt2) : kMaxDirChange;
  if (dt < 0.0) dt = -dt;
  if (dt > kMaxDirChange) dt = kMaxDirChange;
  del *= dt;
  daz *= dt;
  u[0] += del * cos(az) * cos(el) - daz * sin(az);
  u[1] += del * sin(az) * cos(el) + daz * cos(az);
  u[2] -= del * sin(el);
  const double n = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  u[0] /= n; u[1] /= n; u[2] /= n;
  *val = dv[0];
  return dt < kAngleTolerance;
}
template <class SH>
FMLS_HD inline bool get_peak_step(const Tables& t, const SH& sh, double* u, double* val) {
  return newton_step([&](double el, double az, double* dv) { derivatives(t, sh, el, az, dv); }, u, val);
}

// SH::get_peak: at most kPeakSteps Newton steps from u; NaN when it fails.
constexpr int kPeakSteps = 50;
template <class SH>
FMLS_HD inline double get_peak(const Tables& t, const SH& sh, double* u) {
  for (int it = 0; it < kPeakSteps; ++it) {
    double val;
    if (get_peak_step(t, sh, u, &val)) return val;
  }
  u[0] = u[1] = u[2] = NAN;
  return NAN;
}

// FastLookupSet::select_direction (set.cpp:340-354); the grid cell indexes
// are clamped into the grid (a unit vector's z may round a little past 1).
FMLS_HD inline int select_direction(const Tables& t, const double* p) {
  const double az = atan2(p[1], p[0]);
  const double z = p[2] > 1.0 ? 1.0 : (p[2] < -1.0 ? -1.0 : p[2]);
  const double el = acos(z);
  long long ai = (long long)floor((az - t.az_begin) / t.az_step);
  long long ei = (long long)floor((el - t.el_begin) / t.el_step);
  if (ai < 0) ai = 0;
  if (ai >= t.num_az) ai = t.num_az - 1;
  if (ei < 0) ei = 0;
  if (ei >= t.num_el) ei = t.num_el - 1;
  const long long cell = ai * t.num_el + ei;
  int best = t.grid[t.grid_off[cell]];
  double best_dp = fabs(p[0] * t.unit[3 * best] + p[1] * t.unit[3 * best + 1] + p[2] * t.unit[3 * best + 2]);
  for (int e = t.grid_off[cell] + 1; e < t.grid_off[cell + 1]; ++e) {
    const int d = t.grid[e];
    const double dp = fabs(p[0] * t.unit[3 * d] + p[1] * t.unit[3 * d + 1] + p[2] * t.unit[3 * d + 2]);
    if (dp > best_dp) {
      best_dp = dp;
      best = d;
    }
  }
  return best;
}

// fmls.cpp:248-256: the pending ("retrospective") assignments, in order.
template <class W>
FMLS_HD inline void assign_pending(const Tables& t, const W& w, int nr) {
  for (int q = 0; q < nr; ++q) {
    const int d = w.retro_dir[q];
    lobe_add(t, w, root(w, w.retro_lobe[q]), d, w.values[d]);
  }
}

// Whether peak p (created with lobe p) is refined by finish_lobes: its lobe
// (the root of p after the merges) is positive and passes the integral
// threshold (fmls.cpp:258-262).  A peak's starting direction is the one the
// growing left, which finish_lobes changes only after refining that peak, so
// the refinements of all such peaks can be computed beforehand, in parallel.
template <class W>
FMLS_HD inline bool peak_candidate(const Tables& t, const W& w, int p) {
  const int r = root(w, p);
  return !w.neg[r] && !(w.integral[r] < t.integral_threshold);
}

// fmls.cpp:258-301: per surviving lobe (creation order) the thresholds and
// the Newton refinement of its peaks.  pre_val / pre_u (nullable): the
// results of get_peak for every candidate peak p, computed beforehand.
// Writes at most max_out fixels; returns how many lobes survive.
template <class W>
FMLS_HD inline int finish_lobes(const Tables& t, const W& w, const double* sh, int nl, Fixel* out, int max_out,
                                const double* pre_val = nullptr, const double* pre_u = nullptr) {
  int nout = 0;
  for (int r = 0; r < nl; ++r) {
    if (w.parent[r] != r) continue;
    if (w.neg[r] || w.integral[r] < t.integral_threshold) continue;
    int pi = 0;
    for (int p = w.peak_head[r]; p >= 0; p = w.peak_next[p], ++pi) {
      double u[3] = {w.peak_dir[3 * p], w.peak_dir[3 * p + 1], w.peak_dir[3 * p + 2]};
      double val;
      if (pre_val) {
        val = pre_val[p];
        for (int k = 0; k < 3; ++k) u[k] = pre_u[3 * p + k];
      } else {
        val = get_peak(t, sh, u);
      }
      if (!(finite(val) && finite(u[0]) && finite(u[1]) && finite(u[2]))) continue;
      double max_dp = 0.0;
      int nearest = -1, j = 0;
      for (int q = w.peak_head[r]; q >= 0; q = w.peak_next[q], ++j) {
        const double dp = fabs(u[0] * w.peak_dir[3 * q] + u[1] * w.peak_dir[3 * q + 1] + u[2] * w.peak_dir[3 * q + 2]);
        if (dp > max_dp) {
          max_dp = dp;
          nearest = j;
        }
      }
      if (nearest != pi) continue;
      const int c = select_direction(t, u);
      if (w.label[c] < 0 || root(w, w.label[c]) != r) continue;
      for (int k = 0; k < 3; ++k) w.peak_dir[3 * p + k] = u[k];
      if (pi == 0) w.max_peak[r] = val;
    }
    if (w.max_peak[r] < t.peak_value_threshold) continue;
    if (nout < max_out) {
      const double* m = w.mean + 3 * r;
      const double n2 = m[0] * m[0] + m[1] * m[1] + m[2] * m[2];
      const double n = n2 > 0.0 ? sqrt(n2) : 1.0;
      const int h = w.peak_head[r];
      Fixel& f = out[nout];
      for (int k = 0; k < 3; ++k) {
        f.mean_dir[k] = (float)(n2 > 0.0 ? m[k] / n : m[k]);
        f.peak_dir[k] = (float)w.peak_dir[3 * h + k];
      }
      f.integral = (float)w.integral[r];
      f.max_peak = (float)w.max_peak[r];
    }
    ++nout;
  }
  return nout;
}

// fmls.cpp:248-301 after the growing: the pending assignments, then the lobes.
template <class W>
FMLS_HD inline int finish(const Tables& t, const W& w, const double* sh, int nl, int nr, Fixel* out,
                          int max_out) {
  assign_pending(t, w, nr);
  return finish_lobes(t, w, sh, nl, out, max_out);
}

// True when the voxel has no lobes at all (fmls.cpp:166-167, 178-179):
// a DC term that is not positive and finite, a non-finite coefficient, or a
// largest-magnitude amplitude that is not positive (w.order[0] decides).
FMLS_HD inline bool skip_voxel(const double* sh, int nsh) {
  if (!(sh[0] > 0.0) || !finite(sh[0])) return true;
  for (int k = 1; k < nsh; ++k)
    if (!finite(sh[k])) return true;
  return false;
}

}  // namespace fmls
