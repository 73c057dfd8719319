// TEST INFRASTRUCTURE: the FMLS segmentation core (fmls_core.cuh) built for
// the host, so that the CPU tests can compare it with the oracle's literal
// restatement of Segmenter::operator().  Values by plain dot products, the
// order by std::sort with the core's comparator.
#include <algorithm>
#include <cstdint>
#include <vector>

#include <stdexcept>
#include <string>

#include "../include/csd_b200.h"
#include "../mrtrix3_b200/csrc/fmls_core.cuh"
#include "../mrtrix3_b200/csrc/fmls_tables.hpp"

// the library's error recorder and device upload are not compiled into this harness
namespace csdb200 {
int set_error(int code, const std::string&) { return code; }
}
extern "C" int csd_fmls_create(const csd_fmls_tables*, csd_fmls**) { return 0; }

// The C++ table builder's output (csd_fmls_create_default's tables), for
// comparison with the Python host tables: sizes into dims[7], the arrays
// copied into the caller's buffers when they are not null.
extern "C" int fmls_host_default_tables(int lmax, int* dims, double* steps, double* unit, double* weight,
                                        double* sh2amp, double* al, int32_t* adj_off, int32_t* adj,
                                        int32_t* grid_off, int32_t* grid) {
  try {
    const csdb200::FmlsHostTables T = csdb200::build_fmls_tables(lmax);
    dims[0] = T.ndir; dims[1] = T.nsh; dims[2] = T.al_ndir; dims[3] = T.n_al; dims[4] = T.num_az;
    dims[5] = T.num_el; dims[6] = (int)T.grid.size();
    steps[0] = T.al_inc; steps[1] = T.az_begin; steps[2] = T.el_begin; steps[3] = T.az_step; steps[4] = T.el_step;
    if (unit) std::copy(T.unit.begin(), T.unit.end(), unit);
    if (weight) std::copy(T.weight.begin(), T.weight.end(), weight);
    if (sh2amp) std::copy(T.sh2amp.begin(), T.sh2amp.end(), sh2amp);
    if (al) std::copy(T.al.begin(), T.al.end(), al);
    if (adj_off) std::copy(T.adj_off.begin(), T.adj_off.end(), adj_off);
    if (adj) std::copy(T.adj.begin(), T.adj.end(), adj);
    if (grid_off) std::copy(T.grid_off.begin(), T.grid_off.end(), grid_off);
    if (grid) std::copy(T.grid.begin(), T.grid.end(), grid);
    return 0;
  } catch (const std::exception&) {
    return -1;
  }
}

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
