// Oracle test infrastructure only: never linked into, called by, or shipped with the product.
//
// Dual numbers for forward-mode derivatives of the oracle solver (Solver<Dual>): v + d eps with eps^2 = 0.
// Every operation propagates the derivative exactly (up to the rounding of its own arithmetic), so a run
// seeded with d = a perturbation direction yields the directional derivative of its outputs, with no
// finite-difference truncation. Comparisons and branches look at the value only, as the solver's control
// flow does not depend on the derivative.
#ifndef NSF_DUAL_HPP
#define NSF_DUAL_HPP

#include <cmath>

namespace nsfo {

struct Dual {
  double v = 0, d = 0;
  Dual() = default;
  Dual(double x) : v(x), d(0) {}  // NOLINT: implicit, like a double literal
  Dual(double x, double dx) : v(x), d(dx) {}

  Dual& operator+=(const Dual& b) {
    v += b.v;
    d += b.d;
    return *this;
  }
  Dual& operator-=(const Dual& b) {
    v -= b.v;
    d -= b.d;
    return *this;
  }
  Dual& operator*=(const Dual& b) { return *this = Dual(v * b.v, d * b.v + v * b.d); }
  Dual& operator/=(const Dual& b) { return *this = Dual(v / b.v, (d * b.v - v * b.d) / (b.v * b.v)); }
};

inline Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
inline Dual operator+(Dual a, const Dual& b) { return a += b; }
inline Dual operator-(Dual a, const Dual& b) { return a -= b; }
inline Dual operator*(const Dual& a, const Dual& b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(const Dual& a, const Dual& b) { return Dual(a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)); }
inline Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
inline Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
inline Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
inline Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
inline Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
inline Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
inline Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
inline Dual operator/(double a, const Dual& b) { return Dual(a / b.v, -a * b.d / (b.v * b.v)); }

inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }

inline Dual sqrt(const Dual& a) {
  const double s = std::sqrt(a.v);
  return Dual(s, a.d / (2 * s));
}
inline Dual pow(const Dual& a, double e) {
  const double p = std::pow(a.v, e);
  return Dual(p, e * std::pow(a.v, e - 1) * a.d);
}
inline Dual fabs(const Dual& a) { return a.v < 0 ? -a : a; }
inline bool isfinite(const Dual& a) { return std::isfinite(a.v) && std::isfinite(a.d); }

}  // namespace nsfo
#endif
