/* TEST INFRASTRUCTURE ONLY.  Exposes the reference's own
 * MR::Math::Legendre::Plm_sph (core/math/legendre.h:101-123), compiled from
 * the reference source tree by oracle/build_ref.sh, through a C symbol so the
 * oracle's restatement can be compared with it bit for bit. */
#include "math/legendre.h"

namespace {
struct ArrayView {
  using Scalar = double;
  double* p;
  double& operator[](int i) { return p[i]; }
};
}  // namespace

extern "C" void ref_plm_sph(double* out, int lmax, int m, double x) {
  ArrayView a{out};
  MR::Math::Legendre::Plm_sph(a, lmax, m, x);
}
