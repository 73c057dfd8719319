/* Minimal stand-in for MRtrix3's core/math/math.h, providing only the names
 * core/math/legendre.h uses, so that the reference's Legendre recursion can be
 * compiled from its own source without Eigen.  TEST INFRASTRUCTURE ONLY. */
#ifndef ORACLE_REF_STUB_MATH_H
#define ORACLE_REF_STUB_MATH_H
#include <cmath>
#include <cstdlib>
#include <limits>
namespace MR {
namespace Math {
using std::abs;
using std::pow;
constexpr double NaN = std::numeric_limits<double>::quiet_NaN();
template <typename T> inline constexpr T pow2(const T& v) { return v * v; }
}  // namespace Math
}  // namespace MR
#endif
