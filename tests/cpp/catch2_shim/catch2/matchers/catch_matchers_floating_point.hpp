// catch2/matchers/catch_matchers_floating_point.hpp -- the two floating-point
// matchers the reference's tests use, with Catch2 v3's published comparison:
// WithinAbs(t, m) accepts v when t + m >= v and v + m >= t; WithinRel(t, e)
// does the same with the margin e * max(|v|, |t|) (0 if that is infinite), and
// e defaults to 100 epsilons of the target's type.
#pragma once

#include <cmath>
#include <limits>
#include <sstream>
#include <string>

namespace Catch {
namespace Matchers {

namespace shim_detail {
inline bool margin_compare(double lhs, double rhs, double margin) {
  return (lhs + margin >= rhs) && (rhs + margin >= lhs);
}
}  // namespace shim_detail

struct WithinAbsMatcher {
  double target, margin;
  bool match(double v) const { return shim_detail::margin_compare(v, target, margin); }
  std::string describe() const {
    std::ostringstream o;
    o.precision(9);
    o << "is within " << margin << " of " << target;
    return o.str();
  }
};

struct WithinRelMatcher {
  double target, eps;
  bool match(double v) const {
    const double m = eps * std::fmax(std::fabs(v), std::fabs(target));
    return shim_detail::margin_compare(v, target, std::isinf(m) ? 0.0 : m);
  }
  std::string describe() const {
    std::ostringstream o;
    o.precision(9);
    o << "and " << target << " are within " << eps * 100.0 << "% of each other";
    return o.str();
  }
};

inline WithinAbsMatcher WithinAbs(double target, double margin) { return {target, margin}; }
inline WithinRelMatcher WithinRel(double target, double eps) { return {target, eps}; }
inline WithinRelMatcher WithinRel(float target, float eps) { return {target, eps}; }
inline WithinRelMatcher WithinRel(double target) {
  return {target, std::numeric_limits<double>::epsilon() * 100};
}
inline WithinRelMatcher WithinRel(float target) {
  return {target, std::numeric_limits<float>::epsilon() * 100};
}

}  // namespace Matchers
}  // namespace Catch
