// Host-side FP64 precompute of single-shell CSD (the work of MRtrix3's
// CSD::Shared constructor and init(), src/dwi/sdeconv/csd.h:52-198).
// Runs once per gradient scheme on the host; the device only ever sees the
// resulting tables.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace csdb200 {

struct SharedParams {
  int lmax = 0;                 // -lmax (0 = min(lmax_response, 8), csd.h:127)
  int niter = 50;               // -niter (csd.h:35)
  double neg_lambda = 1.0;      // -neg_lambda (csd.h:32)
  double norm_lambda = 1.0;     // -norm_lambda (csd.h:33)
  double threshold = 0.0;       // -threshold (csd.h:34)
  std::vector<double> filter;   // -filter (empty = [1 1 1], csd.h:136-138)
  double bzero_threshold = 10.0;  // BZeroThreshold (dwi/gradient.h:30)
  double bvalue_epsilon = 80.0;   // BValueEpsilon (dwi/shells.h:34)
  std::vector<double> shells;     // -shells b-values (empty = the largest shell, csd.h:64)
};

struct HostShared {
  // sizes
  int lmax = 0, lmax_response = 0, lmax_data = 0;
  int nsh = 0;      // NforL(lmax): FOD coefficients
  int ninit = 0;    // NforL(lmax_response): rows of rconv
  int ndw = 0;      // DW volumes in the selected shell
  int nvol = 0;     // volumes in the gradient table
  int nhr = 0;      // constraint directions
  int niter = 50;
  double neg_lambda = 1.0, norm_lambda = 1.0, threshold = 0.0;
  std::vector<int> dwis;            // [ndw]
  std::vector<double> grad;         // [nvol][4] normalised
  std::vector<double> DW_dirs;      // [ndw][2] az, el
  std::vector<double> rconv;        // [ninit][ndw]
  std::vector<double> M;            // [ndw][nsh]
  std::vector<double> MtM;          // [nsh][nsh], full symmetric, norm_lambda on diag
  std::vector<double> HR;           // [nhr][nsh] HR_trans, scaled
};

// Throws std::runtime_error with the reference's message on invalid input.
HostShared build_shared(const SharedParams& p, const double* grad, int nvol, const double* response,
                        int nresp, const double* hr_dirs, int nhr);

// Exposed for tests of the host library itself.
void plm_sph(double* array, int lmax, int m, double x);
std::vector<double> sh_transform(const double* dirs, int ndir, int lmax);
inline int sh_nforl(int lmax) { return (lmax + 1) * (lmax + 2) / 2; }

}  // namespace csdb200
