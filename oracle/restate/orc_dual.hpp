// Oracle restatement (test infrastructure): forward-mode dual numbers for the FP64 oracle.
//
// `Dual` carries a double value and kDualLanes tangents. Every operation computes its value with
// exactly the double arithmetic that orc::Sim<double> performs (so a Sim<Dual> run takes the same
// branches, contacts, colours and adaptive stops as the Sim<double> run of the same inputs) and
// propagates the tangents by the chain rule. Discrete functions (floor, ceil, comparisons, casts
// to integers) have zero derivative. With the tangents of some inputs seeded, the tangents of the
// outputs are the directional derivatives of the plain FP64 solver: the forward-mode check of the
// hand-written adjoint of the XPBD substep (the active contact set, the colours and the sweep
// counts are those of the value run, as the adjoint freezes them from its forward pass).
#pragma once
#include <cmath>
#include <limits>

namespace orc {

constexpr int kDualLanes = 4;

struct Dual {
  double v = 0.0;
  double d[kDualLanes] = {};
  Dual() = default;
  Dual(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator float() const { return static_cast<float>(v); }
  explicit operator int() const { return static_cast<int>(v); }
  explicit operator long() const { return static_cast<long>(v); }
  explicit operator long long() const { return static_cast<long long>(v); }
  explicit operator unsigned() const { return static_cast<unsigned>(v); }
  explicit operator unsigned long() const { return static_cast<unsigned long>(v); }
  explicit operator unsigned long long() const { return static_cast<unsigned long long>(v); }
  explicit operator unsigned char() const { return static_cast<unsigned char>(v); }
  explicit operator bool() const { return v != 0.0; }
  Dual& operator+=(const Dual& o);
  Dual& operator-=(const Dual& o);
  Dual& operator*=(const Dual& o);
  Dual& operator/=(const Dual& o);
};

// the value and the tangent scale: f(a) with f'(a)
inline Dual chain1(const Dual& a, double f, double df) {
  Dual r(f);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = df * a.d[k];
  return r;
}

inline Dual operator+(const Dual& a, const Dual& b) {
  Dual r(a.v + b.v);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = a.d[k] + b.d[k];
  return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
  Dual r(a.v - b.v);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = a.d[k] - b.d[k];
  return r;
}
inline Dual operator-(const Dual& a) {
  Dual r(-a.v);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = -a.d[k];
  return r;
}
inline Dual operator+(const Dual& a) { return a; }
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r(a.v * b.v);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  Dual r(q);
  for (int k = 0; k < kDualLanes; ++k)
    r.d[k] = (a.d[k] - q * b.d[k]) / b.v;
  return r;
}
inline Dual& Dual::operator+=(const Dual& o) { return *this = *this + o; }
inline Dual& Dual::operator-=(const Dual& o) { return *this = *this - o; }
inline Dual& Dual::operator*=(const Dual& o) { return *this = *this * o; }
inline Dual& Dual::operator/=(const Dual& o) { return *this = *this / o; }

inline bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
inline bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
inline bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
inline bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
inline bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
inline bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }

}  // namespace orc

// the <cmath> functions the oracle calls as std::f(R), for R = Dual
namespace std {
inline orc::Dual sqrt(const orc::Dual& a) {
  const double s = std::sqrt(a.v);
  return orc::chain1(a, s, s > 0.0 ? 0.5 / s : 0.0);
}
inline orc::Dual fabs(const orc::Dual& a) { return a.v < 0.0 ? -a : a; }
inline orc::Dual abs(const orc::Dual& a) { return a.v < 0.0 ? -a : a; }
// fmax / fmin pick an operand (the first on ties, as the value run's result is the same either way)
inline orc::Dual fmax(const orc::Dual& a, const orc::Dual& b) { return (b.v > a.v) ? b : a; }
inline orc::Dual fmin(const orc::Dual& a, const orc::Dual& b) { return (b.v < a.v) ? b : a; }
inline orc::Dual exp(const orc::Dual& a) {
  const double e = std::exp(a.v);
  return orc::chain1(a, e, e);
}
inline orc::Dual log(const orc::Dual& a) { return orc::chain1(a, std::log(a.v), 1.0 / a.v); }
inline orc::Dual sin(const orc::Dual& a) { return orc::chain1(a, std::sin(a.v), std::cos(a.v)); }
inline orc::Dual cos(const orc::Dual& a) { return orc::chain1(a, std::cos(a.v), -std::sin(a.v)); }
inline orc::Dual floor(const orc::Dual& a) { return orc::Dual(std::floor(a.v)); }
inline orc::Dual ceil(const orc::Dual& a) { return orc::Dual(std::ceil(a.v)); }
inline bool isfinite(const orc::Dual& a) { return std::isfinite(a.v); }
inline bool isnan(const orc::Dual& a) { return std::isnan(a.v); }

template <>
class numeric_limits<orc::Dual> {
 public:
  static constexpr bool is_specialized = true;
  static orc::Dual lowest() { return orc::Dual(numeric_limits<double>::lowest()); }
  static orc::Dual max() { return orc::Dual(numeric_limits<double>::max()); }
  static orc::Dual min() { return orc::Dual(numeric_limits<double>::min()); }
  static orc::Dual epsilon() { return orc::Dual(numeric_limits<double>::epsilon()); }
  static orc::Dual infinity() { return orc::Dual(numeric_limits<double>::infinity()); }
};
}  // namespace std
