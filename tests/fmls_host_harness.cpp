// TEST INFRASTRUCTURE: the FMLS segmentation core (fmls_core.cuh) built for
// the host, so that the CPU tests can compare it with the oracle's literal
// restatement of Segmenter::operator().  Values by plain dot products, the
// order by std::sort with the core's comparator.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../include/csd_b200.h"
#include "../mrtrix3_b200/csrc/fmls_core.cuh"

extern "C" int fmls_host_segment(const csd_fmls_tables* c, const double* sh_rows, int n, int max_out,
                                 int32_t* counts, float* fixels) {
  fmls::Tables t{c->ndir, c->lmax, c->nsh, c->unit, c->weight, c->adj_off, c->adj, c->sh2amp,
                 c->al_ndir, c->n_al, c->al_inc, c->al, c->num_az, c->num_el, c->az_begin, c->el_begin,
                 c->az_step, c->el_step, c->grid_off, c->grid, c->integral_threshold, c->peak_value_threshold,
                 c->merge_ratio};
  const int nd = t.ndir;
  std::vector<double> values(nd), mean(3 * nd), integral(nd), max_peak(nd), peak_dir(3 * nd);
  std::vector<int> order(nd), label(nd), parent(nd), neg(nd), head(nd), tail(nd), next(nd), rd(nd), rl(nd);
  fmls::Work w{values.data(), order.data(), label.data(), parent.data(), neg.data(), max_peak.data(),
               mean.data(), integral.data(), head.data(), tail.data(), next.data(), peak_dir.data(), rd.data(),
               rl.data()};
  std::vector<fmls::Fixel> out(max_out);
  for (int v = 0; v < n; ++v) {
    const double* sh = sh_rows + (long long)v * t.nsh;
    counts[v] = 0;
    if (fmls::skip_voxel(sh, t.nsh)) continue;
    for (int d = 0; d < nd; ++d) {
      double s = 0.0;
      for (int k = 0; k < t.nsh; ++k) s += t.sh2amp[(long long)d * t.nsh + k] * sh[k];
      values[d] = s;
      order[d] = d;
    }
    std::sort(order.begin(), order.end(), [&](int a, int b) { return fmls::before(values.data(), nd, a, b); });
    if (values[order[0]] <= 0.0) continue;
    int nr = 0;
    const int nl = fmls::grow(t, w, &nr);
    const int k = fmls::finish(t, w, sh, nl, nr, out.data(), max_out);
    counts[v] = k;
    for (int q = 0; q < std::min(k, max_out); ++q) {
      float* f = fixels + ((long long)v * max_out + q) * 8;
      for (int j = 0; j < 3; ++j) {
        f[j] = out[q].mean_dir[j];
        f[3 + j] = out[q].peak_dir[j];
      }
      f[6] = out[q].integral;
      f[7] = out[q].max_peak;
    }
  }
  return 0;
}
