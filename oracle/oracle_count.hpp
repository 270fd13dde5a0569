// ORACLE (test infrastructure): a counting scalar for the algorithmic FLOP
// count of the restated MHD step.  Counting rules (stated once, used by the
// roofline): add, sub, mul, div and sqrt count 1 each; compare, min, max, abs,
// negation and selects count 0.  Products/sums that the reference evaluates
// through exact-expansion helpers (product_sumN, scaled_product_sum) appear in
// the restatement as their plain N multiplies and N-1 adds, so they are
// counted that way.
#pragma once

#include <cmath>
#include <cstdint>

namespace qoracle {

inline std::uint64_t& flop_counter() {
  static thread_local std::uint64_t n = 0;
  return n;
}

struct Counted {
  double v;
  Counted() : v(0) {}
  Counted(double x) : v(x) {}  // NOLINT: implicit by design (literals)
};

inline Counted operator+(Counted a, Counted b) { ++flop_counter(); return {a.v + b.v}; }
inline Counted operator-(Counted a, Counted b) { ++flop_counter(); return {a.v - b.v}; }
inline Counted operator*(Counted a, Counted b) { ++flop_counter(); return {a.v * b.v}; }
inline Counted operator/(Counted a, Counted b) { ++flop_counter(); return {a.v / b.v}; }
inline Counted operator-(Counted a) { return {-a.v}; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }

inline Counted qsqrt(Counted x) { ++flop_counter(); return {std::sqrt(x.v)}; }
inline Counted qabs(Counted x) { return {std::fabs(x.v)}; }
inline Counted qmin(Counted a, Counted b) { return {std::fmin(a.v, b.v)}; }
inline Counted qmax(Counted a, Counted b) { return {std::fmax(a.v, b.v)}; }
inline bool qfinite(Counted x) { return std::isfinite(x.v); }
inline double qval(Counted x) { return x.v; }

// Counting overloads of the compensated sums: they count as the plain sums
// and products they stand for.
inline Counted crsum(const Counted* t, int n) {
  Counted s = t[0];
  for (int k = 1; k < n; ++k) s = s + t[k];
  return s;
}
inline Counted exact_dot(const double* w, const Counted* x, int n) {
  Counted s = Counted(w[0]) * x[0];
  for (int k = 1; k < n; ++k) s = s + Counted(w[k]) * x[k];
  return s;
}
inline Counted crsum3(Counted a, Counted b, Counted c) { return (a + b) + c; }

}  // namespace qoracle
