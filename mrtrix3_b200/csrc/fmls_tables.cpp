// The FMLS segmenter's tables built on the host from the built-in direction
// set, and csd_fmls_create_default over them.  Restates, for the 1281
// tessellation directions (predefined.cpp, shipped verbatim):
//   Set::initialise (set.h:130-139)            unit vectors from [az el]
//   Segmenter::Segmenter (fmls.cpp:118-140)    SH -> amplitude matrix at the
//                                              [atan2(y, x), acos(z)] of each
//   PrecomputedAL::init (SH.h:416-433)         Legendre table, 2 x 1281 rows
//   FastLookupSet::initialise (set.cpp:365-447) the [az el] lookup grid
// The hull adjacency (set.cpp:83-318) and the integration weights
// (fmls.cpp:87-110) come precomputed from fmls_builtin.inc (generated at
// build time from the data files by the same restatements in Python).
#include "fmls_tables.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include "shared_init.hpp"

namespace csdb200 {
int set_error(int code, const std::string& msg);  // csd_solver.cu
}

namespace {
#include "fmls_builtin.inc"
constexpr double kPi = 3.14159265358979323846;
}  // namespace

namespace csdb200 {

csd_fmls_tables FmlsHostTables::view(double integral_threshold, double peak_value_threshold, double merge_ratio) const {
  csd_fmls_tables t{};
  t.ndir = ndir;
  t.lmax = lmax;
  t.nsh = nsh;
  t.unit = unit.data();
  t.weight = weight.data();
  t.adj_off = adj_off.data();
  t.adj = adj.data();
  t.n_adj = (int)adj.size();
  t.sh2amp = sh2amp.data();
  t.al_ndir = al_ndir;
  t.n_al = n_al;
  t.al_inc = al_inc;
  t.al = al.data();
  t.num_az = num_az;
  t.num_el = num_el;
  t.az_begin = az_begin;
  t.el_begin = el_begin;
  t.az_step = az_step;
  t.el_step = el_step;
  t.grid_off = grid_off.data();
  t.grid = grid.data();
  t.n_grid = (int)grid.size();
  t.integral_threshold = integral_threshold;
  t.peak_value_threshold = peak_value_threshold;
  t.merge_ratio = merge_ratio;
  return t;
}

FmlsHostTables build_fmls_tables(int lmax) {
  if (lmax < 0 || lmax > 16 || (lmax & 1)) throw std::runtime_error("lmax must be even and at most 16");
  FmlsHostTables T;
  const int nd = (int)(sizeof(kTess1281Weight) / sizeof(double));
  T.lmax = lmax;
  T.nsh = sh_nforl(lmax);
  T.ndir = nd;
  T.unit.resize(3 * (size_t)nd);
  for (int i = 0; i < nd; ++i) {
    const double az = kTess1281AzEl[2 * i], el = kTess1281AzEl[2 * i + 1], s = std::sin(el);
    T.unit[3 * i] = std::cos(az) * s;
    T.unit[3 * i + 1] = std::sin(az) * s;
    T.unit[3 * i + 2] = std::cos(el);
  }
  T.weight.assign(kTess1281Weight, kTess1281Weight + nd);
  T.adj_off.assign(kTess1281AdjOff, kTess1281AdjOff + nd + 1);
  T.adj.assign(kTess1281Adj, kTess1281Adj + T.adj_off[nd]);
  // SH -> amplitudes at the directions' own [az el]
  std::vector<double> azel(2 * (size_t)nd);
  for (int i = 0; i < nd; ++i) {
    azel[2 * i] = std::atan2(T.unit[3 * i + 1], T.unit[3 * i]);
    azel[2 * i + 1] = std::acos(T.unit[3 * i + 2]);
  }
  T.sh2amp = sh_transform(azel.data(), nd, lmax);
  // PrecomputedAL with 2 ndir elevations
  T.al_ndir = 2 * nd;
  T.n_al = (lmax / 2 + 1) * (lmax / 2 + 1);
  T.al_inc = kPi / (T.al_ndir - 1);
  T.al.assign((size_t)T.al_ndir * T.n_al, 0.0);
  std::vector<double> buf(lmax + 2);
  for (int n = 0; n < T.al_ndir; ++n) {
    const double z = std::cos(n * T.al_inc);
    for (int m = 0; m <= lmax; ++m) {
      plm_sph(buf.data(), lmax, m, z);
      for (int l = (m & 1) ? m + 1 : m; l <= lmax; l += 2) T.al[(size_t)n * T.n_al + l * l / 4 + m] = buf[l];
    }
  }
  // FastLookupSet grid
  double sum = 0.0;
  long long count = 0;
  for (int i = 0; i < nd; ++i)
    for (int e = T.adj_off[i]; e < T.adj_off[i + 1]; ++e) {
      const int j = T.adj[e];
      if (j > i) {
        sum += std::fabs(T.unit[3 * i] * T.unit[3 * j] + T.unit[3 * i + 1] * T.unit[3 * j + 1] +
                         T.unit[3 * i + 2] * T.unit[3 * j + 2]);
        ++count;
      }
    }
  const double step = std::acos(sum / (double)count);
  T.num_az = (int)std::ceil(2.0 * kPi / step);
  T.num_el = (int)std::ceil(kPi / step);
  T.az_step = 2.0 * kPi / (double)(T.num_az - 1);
  T.el_step = kPi / (double)(T.num_el - 1);
  T.az_begin = -kPi;
  T.el_begin = 0.0;
  const int ncell = T.num_az * T.num_el;
  std::vector<std::vector<int32_t>> cells(ncell);
  auto cell_of = [&](const double* p) {
    const double az = std::atan2(p[1], p[0]), el = std::acos(p[2]);
    return (long long)std::floor((az - T.az_begin) / T.az_step) * T.num_el +
           (long long)std::floor((el - T.el_begin) / T.el_step);
  };
  for (int i = 0; i < nd; ++i) {
    const long long c = cell_of(&T.unit[3 * i]);
    if (c < 0 || c >= ncell) throw std::runtime_error("direction outside the lookup grid");
    cells[c].push_back(i);
  }
  for (int c = 0; c < ncell; ++c) {
    const int ai = c / T.num_el, ei = c - ai * T.num_el;
    for (int corner = 0; corner < 4; ++corner) {
      double az = T.az_begin + ai * T.az_step, el = T.el_begin + ei * T.el_step;
      if (corner == 1 || corner == 2) az += T.az_step;
      if (corner == 2 || corner == 3) el += T.el_step;
      const double p[3] = {std::cos(az) * std::sin(el), std::sin(az) * std::sin(el), std::cos(el)};
      int best = 0;
      double best_dp = std::fabs(p[0] * T.unit[0] + p[1] * T.unit[1] + p[2] * T.unit[2]);
      for (int d = 1; d < nd; ++d) {
        const double dp = std::fabs(p[0] * T.unit[3 * d] + p[1] * T.unit[3 * d + 1] + p[2] * T.unit[3 * d + 2]);
        if (dp > best_dp) {
          best_dp = dp;
          best = d;
        }
      }
      if (std::find(cells[c].begin(), cells[c].end(), best) == cells[c].end()) cells[c].push_back(best);
    }
  }
  for (auto& cell : cells) {
    const size_t n0 = cell.size();
    for (size_t q = 0; q < n0; ++q) {
      const int d = cell[q];
      for (int e = T.adj_off[d]; e < T.adj_off[d + 1]; ++e)
        if (std::find(cell.begin(), cell.end(), T.adj[e]) == cell.end()) cell.push_back(T.adj[e]);
    }
    std::sort(cell.begin(), cell.end());
  }
  T.grid_off.assign(1, 0);
  for (const auto& cell : cells) {
    T.grid.insert(T.grid.end(), cell.begin(), cell.end());
    T.grid_off.push_back((int32_t)T.grid.size());
  }
  return T;
}

}  // namespace csdb200

extern "C" int csd_fmls_create_default(int lmax, double integral_threshold, double peak_value_threshold,
                                       double merge_ratio, csd_fmls** out) {
  if (!out) return csdb200::set_error(CSD_ERR_INVALID, "csd_fmls_create_default: null argument");
  *out = nullptr;
  try {
    const csdb200::FmlsHostTables T = csdb200::build_fmls_tables(lmax);
    const csd_fmls_tables t = T.view(integral_threshold, peak_value_threshold, merge_ratio);
    return csd_fmls_create(&t, out);  // copies the tables to the device
  } catch (const std::exception& e) {
    return csdb200::set_error(CSD_ERR_INVALID, std::string("csd_fmls_create_default: ") + e.what());
  }
}
