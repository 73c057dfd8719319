// Host tables of fod2fixel's FMLS segmenter on the built-in 1281-direction
// set (FMLS::Segmenter's constructor, src/dwi/fmls.cpp:118-140).
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/csd_b200.h"

namespace csdb200 {

struct FmlsHostTables {
  int lmax = 0, nsh = 0, ndir = 0, al_ndir = 0, n_al = 0, num_az = 0, num_el = 0;
  double al_inc = 0, az_begin = 0, el_begin = 0, az_step = 0, el_step = 0;
  std::vector<double> unit, weight, sh2amp, al;
  std::vector<int32_t> adj_off, adj, grid_off, grid;
  csd_fmls_tables view(double integral_threshold, double peak_value_threshold, double merge_ratio) const;
};

// Throws std::runtime_error for an lmax outside 0..16 or odd.
FmlsHostTables build_fmls_tables(int lmax);

}  // namespace csdb200
