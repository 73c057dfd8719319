// FP64 host precompute for single-shell CSD.  Follows MRtrix3
// src/dwi/sdeconv/csd.h:52-198 and the helpers it calls; every step cites the
// reference lines it mirrors.
#include "shared_init.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>

namespace csdb200 {
namespace {

int sh_index(int l, int m) { return l * (l + 1) / 2 + m; }  // SH.h:52-55

// SH.h:70-73 (the square root is taken in single precision upstream)
int sh_lforn(int n) {
  if (!n) return 0;
  return 2 * static_cast<int>(std::floor((std::sqrt(static_cast<float>(1 + 8 * n)) - 3.0) / 4.0));
}
int zsh_nforl(int lmax) { return 1 + lmax / 2; }  // ZSH.h:42-45
int zsh_lforn(int n) { return 2 * (n - 1); }       // ZSH.h:54-57

double helper(double x, double m) {  // legendre.h:66-70
  return m < 1.0 ? 1.0 : x * (m - 1.0) / m * helper(x, m - 2.0);
}

// Dense Cholesky of a symmetric positive definite matrix (row-major, lower).
bool cholesky(std::vector<double>& A, int n) {
  for (int j = 0; j < n; ++j) {
    double d = A[j * n + j];
    for (int k = 0; k < j; ++k) d -= A[j * n + k] * A[j * n + k];
    if (!(d > 0.0)) return false;
    d = std::sqrt(d);
    A[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double s = A[i * n + j];
      for (int k = 0; k < j; ++k) s -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = s / d;
    }
  }
  return true;
}
void cholesky_solve(const std::vector<double>& L, int n, double* x) {
  for (int i = 0; i < n; ++i) {
    double s = x[i];
    for (int k = 0; k < i; ++k) s -= L[i * n + k] * x[k];
    x[i] = s / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = x[i];
    for (int k = i + 1; k < n; ++k) s -= L[k * n + i] * x[k];
    x[i] = s / L[i * n + i];
  }
}

// A b-value shell as Shell::Shell (dwi/shells.cpp:52-70) describes it: mean,
// sample standard deviation, min and -- as computed there -- "max", the
// larger of the running minimum and the last volume's b.
struct Shell {
  double mean, stdev, lo, hi;
  std::vector<int> vols;
  bool is_bzero(double b0thr) const { return mean <= b0thr; }
};

// dwi/shells.cpp:347-411 (clustering) + :300-345 (shell construction):
// the shells by increasing mean b-value.
std::vector<Shell> cluster_shells(const std::vector<double>& b, double b0thr, double eps) {
  const int nvol = static_cast<int>(b.size());
  std::vector<int> clusters(nvol, 0);
  std::vector<char> visited(nvol, 0);
  auto region = [&](double bv, std::vector<int>& idx) {
    for (int i = 0; i < nvol; ++i)
      if (b[i] > b0thr && std::fabs(bv - b[i]) < eps) idx.push_back(i);
  };
  int cluster = 0;
  for (int i = 0; i < nvol; ++i)
    if (b[i] <= b0thr) {
      visited[i] = 1;
      cluster = 1;
      clusters[i] = 1;
    }
  for (int i = 0; i < nvol; ++i) {
    if (visited[i]) continue;
    visited[i] = 1;
    std::vector<int> nb;
    region(b[i], nb);
    if (b[i] > b0thr && nb.size() < 3) {
      clusters[i] = 0;
      continue;
    }
    clusters[i] = ++cluster;
    for (size_t q = 0; q < nb.size(); ++q) {
      const int v = nb[q];
      if (!visited[v]) {
        visited[v] = 1;
        std::vector<int> nb2;
        region(b[v], nb2);
        if (nb2.size() >= 3)
          for (int x : nb2) nb.push_back(x);
      }
      if (clusters[v] == 0) clusters[v] = cluster;
    }
  }
  const int nshells = cluster;
  if (nshells < 1 || nshells > std::sqrt(static_cast<double>(nvol)))
    throw std::runtime_error(
        "DWI volumes could not be classified into b-value shells; gradient encoding may not represent a "
        "HARDI sequence");
  std::vector<Shell> shells;
  for (int s = 1; s <= nshells; ++s) {
    Shell sh{0.0, 0.0, std::numeric_limits<double>::max(), 0.0, {}};
    for (int v = 0; v < nvol; ++v)
      if (clusters[v] == s) {
        sh.vols.push_back(v);
        sh.mean += b[v];
        sh.lo = std::min(sh.lo, b[v]);
        sh.hi = std::max(sh.lo, b[v]);
      }
    if (sh.vols.empty()) continue;
    sh.mean /= sh.vols.size();
    for (int v : sh.vols) sh.stdev += (b[v] - sh.mean) * (b[v] - sh.mean);
    sh.stdev = std::sqrt(sh.stdev / (static_cast<double>(sh.vols.size()) - 1.0));
    shells.push_back(std::move(sh));
  }
  std::stable_sort(shells.begin(), shells.end(), [](const Shell& a, const Shell& c) { return a.mean < c.mean; });
  return shells;
}

std::string shell_str(const Shell& s) {
  std::ostringstream o;
  o << s.mean << " +- " << s.stdev;
  return o.str();
}

// csd.h:62-64: Shells(grad).select_shells(true, false, true).largest() --
// the volumes of the one non-b=0 shell CSD uses.  Without -shells
// (n_req == 0) that is the largest b-value shell (dwi/shells.cpp:243-260);
// with it, the shells matching the requested b-values (dwi/shells.cpp:111-239)
// must be exactly one non-b=0 shell and no b=0 shell.
std::vector<int> csd_shell(const std::vector<double>& b, double b0thr, double eps, const double* req, int n_req) {
  std::vector<Shell> shells = cluster_shells(b, b0thr, eps);
  const bool has_b0 = shells.front().is_bzero(b0thr);
  if (n_req <= 0) {
    if (shells.size() == 1 && has_b0)
      throw std::runtime_error("No non b=0 data found, but the command requires a non b=0 shell");
    return shells.back().vols;
  }
  std::vector<char> keep(shells.size(), 0);
  bool b0_selected = false;
  int nonb0_selected = 0;
  auto take = [&](size_t s) {
    if (keep[s])
      throw std::runtime_error("User selected a shell more than once: " + shell_str(shells[s]) + " with " +
                               std::to_string(shells[s].vols.size()) + " volumes");
    keep[s] = 1;
    ++nonb0_selected;
  };
  for (int q = 0; q < n_req; ++q) {
    const double want = req[q];
    if (want < 0.0) throw std::runtime_error("Cannot select shells corresponding to negative b-values");
    if (want <= b0thr) {
      if (!has_b0) throw std::runtime_error("User selected b=0 shell, but no such data was found");
      if (b0_selected) throw std::runtime_error("User selected b=0 shell more than once");
      keep[0] = 1;
      b0_selected = true;
      continue;
    }
    // within a shell's [min, "max"] range
    bool selected = false;
    for (size_t s = 0; s < shells.size(); ++s)
      if (want >= shells[s].lo && want <= shells[s].hi) {
        take(s);
        selected = true;
      }
    if (selected) continue;
    // within 1 of exactly one shell's mean
    size_t best = 0;
    bool ambiguous = false;
    for (size_t s = 0; s < shells.size(); ++s)
      if (std::fabs(want - shells[s].mean) <= 1.0) {
        if (selected) {
          ambiguous = true;
        } else {
          best = s;
          selected = true;
        }
      }
    if (selected && !ambiguous) {
      take(best);
      continue;
    }
    // the clear winner in standard deviations (Poisson when a non-b=0 shell
    // has a negligible spread)
    bool zero_stdev = false;
    for (const Shell& s : shells)
      if (!s.is_bzero(b0thr) && s.stdev < 1.0) zero_stdev = true;
    best = 0;
    double best_n = std::numeric_limits<double>::max();
    ambiguous = false;
    for (size_t s = 0; s < shells.size(); ++s) {
      const double sd = shells[s].is_bzero(b0thr) ? 0.5 * b0thr
                                                  : (zero_stdev ? std::sqrt(shells[s].mean) : shells[s].stdev);
      const double n = std::fabs((want - shells[s].mean) / sd);
      if (n < best_n) {
        ambiguous = n >= 0.1 * best_n;
        best = s;
        best_n = n;
      } else {
        ambiguous = n < 10.0 * best_n;
      }
    }
    if (ambiguous) {
      std::string all;
      for (const Shell& s : shells) all += (all.empty() ? "" : ", ") + shell_str(s);
      std::ostringstream o;
      o << "Unable to robustly select desired shell b=" << want << " (detected shells are: " << all << ")";
      throw std::runtime_error(o.str());
    }
    take(best);
  }
  if (nonb0_selected != 1)
    throw std::runtime_error("User selected " + std::to_string(nonb0_selected) +
                             " non b=0 shells, but the command requires single-shell data");
  if (b0_selected) throw std::runtime_error("User selected b=0 shell, but the command is not compatible with b=0 data");
  for (size_t s = shells.size(); s-- > 0;)
    if (keep[s]) return shells[s].vols;
  throw std::runtime_error("no shell selected");
}

}  // namespace

// legendre.h:101-123
void plm_sph(double* a, int lmax, int m, double x) {
  const double x2 = x * x;
  if (m && x2 >= 1.0) {
    for (int n = m; n <= lmax; ++n) a[n] = 0.0;
    return;
  }
  a[m] = 0.282094791773878;
  if (m) a[m] *= std::sqrt(static_cast<double>(2 * m + 1) * helper(1.0 - x2, 2.0 * m));
  if (m & 1) a[m] = -a[m];
  if (lmax == m) return;
  double f = std::sqrt(static_cast<double>(2 * m + 3));
  a[m + 1] = x * f * a[m];
  for (int n = m + 2; n <= lmax; ++n) {
    a[n] = x * a[n - 1] - a[n - 2] / f;
    f = std::sqrt(static_cast<double>(4 * n * n - 1) / static_cast<double>(n * n - m * m));
    a[n] *= f;
  }
}

// SH.h:82-104
std::vector<double> sh_transform(const double* dirs, int ndir, int lmax) {
  const int N = sh_nforl(lmax);
  std::vector<double> T(static_cast<size_t>(ndir) * N, 0.0);
  std::vector<double> AL(lmax + 2);
  const double sqrt2 = std::sqrt(2.0);
  for (int i = 0; i < ndir; ++i) {
    double* row = &T[static_cast<size_t>(i) * N];
    const double az = dirs[2 * i], z = std::cos(dirs[2 * i + 1]);
    plm_sph(AL.data(), lmax, 0, z);
    for (int l = 0; l <= lmax; l += 2) row[sh_index(l, 0)] = AL[l];
    for (int m = 1; m <= lmax; ++m) {
      plm_sph(AL.data(), lmax, m, z);
      for (int l = (m & 1) ? m + 1 : m; l <= lmax; l += 2) {
        row[sh_index(l, m)] = sqrt2 * AL[l] * std::cos(m * az);
        row[sh_index(l, -m)] = sqrt2 * AL[l] * std::sin(m * az);
      }
    }
  }
  return T;
}

HostShared build_shared(const SharedParams& p, const double* grad_in, int nvol, const double* response,
                        int nresp, const double* hr_dirs, int nhr) {
  if (nvol <= 0 || !grad_in) throw std::runtime_error("empty gradient table");
  if (nresp <= 0 || !response) throw std::runtime_error("empty response function");
  if (nhr <= 0 || !hr_dirs) throw std::runtime_error("empty constraint direction set");
  HostShared s;
  s.nvol = nvol;
  s.nhr = nhr;
  s.niter = p.niter;
  if (p.niter < 0) throw std::runtime_error("niter must be non-negative");

  // dwi/gradient.cpp:286-310: normalise directions; scale b by |g|^2 when the
  // norms stray from 1 by more than exp(0.01)
  s.grad.assign(grad_in, grad_in + 4 * static_cast<size_t>(nvol));
  std::vector<double> sq(nvol);
  double maxlog = 0.0;
  for (int r = 0; r < nvol; ++r) {
    double* g = &s.grad[4 * r];
    sq[r] = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
    if (sq[r]) {
      const double n = std::sqrt(sq[r]);
      g[0] /= n;
      g[1] /= n;
      g[2] /= n;
    }
    maxlog = std::max(maxlog, sq[r] > 0.0 ? std::fabs(std::log(sq[r])) : 0.0);
  }
  if (maxlog > 0.01)
    for (int r = 0; r < nvol; ++r) s.grad[4 * r + 3] *= sq[r];

  // csd.h:62-64: volumes of the largest non-b=0 shell
  std::vector<double> b(nvol);
  for (int r = 0; r < nvol; ++r) b[r] = s.grad[4 * r + 3];
  s.dwis = csd_shell(b, p.bzero_threshold, p.bvalue_epsilon, p.shells.data(), static_cast<int>(p.shells.size()));
  s.ndw = static_cast<int>(s.dwis.size());

  // gradient.h:77-95
  s.DW_dirs.resize(2 * static_cast<size_t>(s.ndw));
  for (int i = 0; i < s.ndw; ++i) {
    const double* g = &s.grad[4 * s.dwis[i]];
    s.DW_dirs[2 * i] = std::atan2(g[1], g[0]);
    const double z = g[2] / std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    s.DW_dirs[2 * i + 1] = z >= 1.0 ? 0.0 : (z <= -1.0 ? M_PI : std::acos(z));
  }

  s.lmax_data = sh_lforn(s.ndw);            // csd.h:67
  int lmax_response = zsh_lforn(nresp);     // csd.h:112
  if (s.lmax_data <= 0) throw std::runtime_error("data contain too few directions even for lmax = 2");
  if (lmax_response <= 0) throw std::runtime_error("response function does not contain anisotropic terms");
  s.lmax = p.lmax ? p.lmax : std::min(lmax_response, 8);  // csd.h:127
  if (s.lmax <= 0 || s.lmax % 2) throw std::runtime_error("lmax must be a positive even integer");
  lmax_response = std::min(lmax_response, std::min(s.lmax_data, s.lmax));  // csd.h:133
  s.lmax_response = lmax_response;
  s.nsh = sh_nforl(s.lmax);
  s.ninit = sh_nforl(lmax_response);

  // csd.h:136-138
  std::vector<double> filt(zsh_nforl(lmax_response), 0.0);
  if (p.filter.empty()) {
    for (size_t i = 0; i < filt.size() && i < 3; ++i) filt[i] = 1.0;
  } else {
    for (size_t i = 0; i < filt.size() && i < p.filter.size(); ++i) filt[i] = p.filter[i];
  }
  // csd.h:140-142, ZSH.h:221-231
  std::vector<double> RH(std::max<int>(zsh_nforl(s.lmax), nresp), 0.0);
  {
    const int lr = zsh_lforn(nresp);
    std::vector<double> AL(lr + 2);
    plm_sph(AL.data(), lr, 0, 1.0);
    for (int l = 0; l <= lr; l += 2) RH[l / 2] = response[l / 2] / AL[l];
  }

  // csd.h:145-158: rconv = pinv(fconv with 1e-2 added to its (i,i) entries)
  {
    const int nr = s.ninit, ndw = s.ndw;
    if (ndw < nr) throw std::runtime_error("fewer DW directions than initialisation coefficients");
    std::vector<double> fconv = sh_transform(s.DW_dirs.data(), ndw, lmax_response);
    for (int i = 0; i < std::min(ndw, nr); ++i) fconv[i * nr + i] += 1.0e-2;
    std::vector<double> FtF(static_cast<size_t>(nr) * nr);
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nr; ++j) {
        double acc = 0.0;
        for (int k = 0; k < ndw; ++k) acc += fconv[k * nr + i] * fconv[k * nr + j];
        FtF[i * nr + j] = acc;
      }
    if (!cholesky(FtF, nr)) throw std::runtime_error("pinv: normal matrix not positive definite");
    s.rconv.assign(static_cast<size_t>(nr) * ndw, 0.0);
    std::vector<double> col(nr);
    for (int k = 0; k < ndw; ++k) {
      for (int i = 0; i < nr; ++i) col[i] = fconv[k * nr + i];
      cholesky_solve(FtF, nr, col.data());
      for (int i = 0; i < nr; ++i) s.rconv[i * ndw + k] = col[i];
    }
    int l = 0, nl = 1;
    for (int row = 0; row < nr; ++row) {
      if (row >= nl) {
        ++l;
        nl = sh_nforl(2 * l);
      }
      const double sc = filt[l] / RH[l];
      for (int k = 0; k < ndw; ++k) s.rconv[row * ndw + k] *= sc;
    }
  }

  // csd.h:163-172, 184-188
  s.M = sh_transform(s.DW_dirs.data(), s.ndw, s.lmax);
  {
    int l = 0, nl = 1;
    for (int c = 0; c < s.nsh; ++c) {
      if (c >= nl) {
        ++l;
        nl = sh_nforl(2 * l);
      }
      for (int k = 0; k < s.ndw; ++k) s.M[k * s.nsh + c] *= RH[l];
    }
  }

  // csd.h:175-180
  s.HR = sh_transform(hr_dirs, nhr, s.lmax);
  const double cm = p.neg_lambda * 50.0 * response[0] / static_cast<double>(nhr);
  for (double& v : s.HR) v *= cm;
  s.threshold = p.threshold * cm;
  s.neg_lambda = p.neg_lambda;

  // csd.h:188-195
  const int n = s.nsh;
  s.MtM.assign(static_cast<size_t>(n) * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double acc = 0.0;
      for (int k = 0; k < s.ndw; ++k) acc += s.M[k * n + i] * s.M[k * n + j];
      s.MtM[i * n + j] = acc;
      s.MtM[j * n + i] = acc;
    }
  s.norm_lambda = p.norm_lambda;
  if (p.norm_lambda) {
    s.norm_lambda = p.norm_lambda * 0.0002 * s.MtM[0];
    for (int i = 0; i < n; ++i) s.MtM[i * n + i] += s.norm_lambda;
  }
  return s;
}

}  // namespace csdb200
