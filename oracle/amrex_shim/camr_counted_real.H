// A double that counts the floating-point operations done on it: the
// AMReX stand-in's amrex::Real when CAMR_FLOP_COUNT is defined, so that the
// reference's own hydro sources, compiled unmodified, report how many
// operations one box of the hydro performs (the algorithmic flop count of
// the measurement).  Counted as flops: +, -, *, / and sqrt (one each);
// counted apart and not as flops: comparisons, min/max, abs, copysign.
// Test infrastructure only (oracle/flops.cpp).
#pragma once

#include <algorithm>
#include <cmath>

namespace camr_flops {

struct Counts {
  long long add = 0, mul = 0, div = 0, sqrt = 0, cmp = 0, other = 0;
};
inline Counts& counts() {
  static thread_local Counts c;
  return c;
}

struct CountedReal {
  double v;
  CountedReal() = default;
  constexpr CountedReal(double x) : v(x) {}  // NOLINT: literals and doubles convert implicitly
  explicit operator double() const { return v; }
  CountedReal& operator+=(CountedReal o) { ++counts().add; v += o.v; return *this; }
  CountedReal& operator-=(CountedReal o) { ++counts().add; v -= o.v; return *this; }
  CountedReal& operator*=(CountedReal o) { ++counts().mul; v *= o.v; return *this; }
  CountedReal& operator/=(CountedReal o) { ++counts().div; v /= o.v; return *this; }
};

inline CountedReal operator+(CountedReal a, CountedReal b) { ++counts().add; return a.v + b.v; }
inline CountedReal operator-(CountedReal a, CountedReal b) { ++counts().add; return a.v - b.v; }
inline CountedReal operator*(CountedReal a, CountedReal b) { ++counts().mul; return a.v * b.v; }
inline CountedReal operator/(CountedReal a, CountedReal b) { ++counts().div; return a.v / b.v; }
inline CountedReal operator-(CountedReal a) { return -a.v; }
inline CountedReal operator+(CountedReal a) { return a; }
inline bool operator<(CountedReal a, CountedReal b) { ++counts().cmp; return a.v < b.v; }
inline bool operator>(CountedReal a, CountedReal b) { ++counts().cmp; return a.v > b.v; }
inline bool operator<=(CountedReal a, CountedReal b) { ++counts().cmp; return a.v <= b.v; }
inline bool operator>=(CountedReal a, CountedReal b) { ++counts().cmp; return a.v >= b.v; }
inline bool operator==(CountedReal a, CountedReal b) { ++counts().cmp; return a.v == b.v; }
inline bool operator!=(CountedReal a, CountedReal b) { ++counts().cmp; return a.v != b.v; }

inline CountedReal abs(CountedReal a) { ++counts().other; return std::fabs(a.v); }
inline CountedReal copysign(CountedReal a, CountedReal b) {
  ++counts().other;
  return std::copysign(a.v, b.v);
}
inline CountedReal sqrt(CountedReal a) { ++counts().sqrt; return std::sqrt(a.v); }

}  // namespace camr_flops

namespace std {
// std::min / std::max with the reference's mixed double / Real arguments
// (std's templates need one type); first argument wins ties, as std's do.
inline camr_flops::CountedReal min(camr_flops::CountedReal a, camr_flops::CountedReal b) {
  return (b < a) ? b : a;
}
inline camr_flops::CountedReal max(camr_flops::CountedReal a, camr_flops::CountedReal b) {
  return (a < b) ? b : a;
}
inline camr_flops::CountedReal abs(camr_flops::CountedReal a) { return camr_flops::abs(a); }
inline camr_flops::CountedReal sqrt(camr_flops::CountedReal a) { return camr_flops::sqrt(a); }
inline camr_flops::CountedReal copysign(camr_flops::CountedReal a, camr_flops::CountedReal b) {
  return camr_flops::copysign(a, b);
}
}  // namespace std
