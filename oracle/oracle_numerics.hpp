// ORACLE (test infrastructure, never shipped): CPU restatement of the
// reference's pointwise ideal-MHD numerics, following the reference formula by
// formula in ordinary binary64 arithmetic.  Every function cites the
// reference file:line it restates (paths relative to the quasar tree).
//
// The reference evaluates most sums of products through exact-expansion
// "scaled" arithmetic (include/quasar/numerics/scaled_arithmetic.hpp:121-308):
// correctly rounded sums that also keep intermediates out of binary64
// overflow.  This restatement evaluates the same sums with compensated
// (Sum2/Dot2) arithmetic at the same call sites, which reproduces the rounded
// results except in rare ties, and plain IEEE arithmetic elsewhere; it does
// not restate the overflow protection (states here are O(1e-6..1e6)).  The
// remaining rounding-level differences are pinned by
// tests/test_oracle_vs_reference.py.
//
// Everything is templated on the scalar R.  R = double is the oracle;
// R = Counted (oracle_count.hpp) counts algorithmic FLOPs under the rules:
// + - * / sqrt = 1, compare/min/max/abs = 0.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

namespace qoracle {

// ---- scalar helpers (overloaded for Counted in oracle_count.hpp) ----------
inline double qsqrt(double x) { return std::sqrt(x); }
inline double qabs(double x) { return std::fabs(x); }
inline double qmin(double a, double b) { return std::fmin(a, b); }
inline double qmax(double a, double b) { return std::fmax(a, b); }
inline bool qfinite(double x) { return std::isfinite(x); }
inline double qval(double x) { return x; }

// Compensated sums standing in for the reference's exact-expansion reductions
// (scaled_arithmetic.hpp:121-286).  crsum: sum of already-rounded terms with
// the TwoSum error carried (Ogita-Rump-Oishi Sum2), which returns the correctly
// rounded sum except in rare double-rounding ties.  exact_dot: the same with
// error-free FMA products (Dot2), used where the reference forms exact
// coefficient*sample products (append_scaled_exact_product,
// scaled_arithmetic.hpp:447-481).  Exactness matters: e.g. a constant field
// collocates to itself bit for bit, and E + v^2/2 - v^2/2 returns E.
inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
inline double crsum(const double* t, int n) {
  double s = t[0], c = 0.0;
  for (int k = 1; k < n; ++k) {
    double e;
    two_sum(s, t[k], s, e);
    c += e;
  }
  return s + c;
}
inline double exact_dot(const double* w, const double* x, int n) {
  double s = w[0] * x[0];
  double c = std::fma(w[0], x[0], -s);
  for (int k = 1; k < n; ++k) {
    const double p = w[k] * x[k];
    const double pe = std::fma(w[k], x[k], -p);
    double e;
    two_sum(s, p, s, e);
    c += e + pe;
  }
  return s + c;
}
inline double crsum3(double a, double b, double c) {
  const double t[3] = {a, b, c};
  return crsum(t, 3);
}

constexpr double kEps = std::numeric_limits<double>::epsilon();
constexpr double kTiny = std::numeric_limits<double>::min();

template <class R>
struct State {
  R rho, mx, my, mz, energy, bx, by, bz;
};
template <class R>
struct Prim {
  R rho, vx, vy, vz, p, bx, by, bz;
};

// mhd_state.hpp:92-100
template <class R>
R scaled_norm3(R x, R y, R z) {
  const R scale = qmax(qabs(x), qmax(qabs(y), qabs(z)));
  if (scale == R(0)) return R(0);
  const R xs = x / scale, ys = y / scale, zs = z / scale;
  return scale * qsqrt(xs * xs + ys * ys + zs * zs);
}

// mhd_state.hpp:105-114
template <class R>
R half_squared_norm3(R x, R y, R z) {
  const R scale = qmax(qabs(x), qmax(qabs(y), qabs(z)));
  if (scale == R(0)) return R(0);
  const R xs = x / scale, ys = y / scale, zs = z / scale;
  const R n2 = xs * xs + ys * ys + zs * zs;
  return (R(0.5) * scale) * (scale * n2);
}

// mhd_state.hpp:118-128
template <class R>
R kinetic_from_momentum(R mx, R my, R mz, R rho) {
  const R scale = qmax(qabs(mx), qmax(qabs(my), qabs(mz)));
  if (scale == R(0)) return R(0);
  const R xs = mx / scale, ys = my / scale, zs = mz / scale;
  const R q = scale / qsqrt(rho);
  const R n2 = xs * xs + ys * ys + zs * zs;
  return (R(0.5) * q) * (q * n2);
}

// mhd_state.hpp:131-141
template <class R>
R kinetic_from_velocity(R rho, R vx, R vy, R vz) {
  const R scale = qmax(qabs(vx), qmax(qabs(vy), qabs(vz)));
  if (scale == R(0)) return R(0);
  const R xs = vx / scale, ys = vy / scale, zs = vz / scale;
  const R q = qsqrt(rho) * scale;
  const R n2 = xs * xs + ys * ys + zs * zs;
  return (R(0.5) * q) * (q * n2);
}

// mhd_state.hpp:148-182 (dir selects the normal Alfven component)
template <class R>
void magnetosonic_speeds(R rho, R p, R bx, R by, R bz, int dir, R gamma,
                         R& fast, R& slow, R& sound, R& can_out, R& ca_out) {
  const R sqrt_rho = qsqrt(rho);
  sound = (p > R(0) && gamma > R(0)) ? qsqrt(gamma) * (qsqrt(p) / sqrt_rho)
                                     : R(0);
  const R ax = bx / sqrt_rho, ay = by / sqrt_rho, az = bz / sqrt_rho;
  ca_out = scaled_norm3(ax, ay, az);
  can_out = qabs(dir == 0 ? ax : ay);
  const R scale = qmax(sound, ca_out);
  if (!(scale > R(0))) {
    fast = R(0);
    slow = R(0);
    return;
  }
  const R an = sound / scale, bn = ca_out / scale, cn = can_out / scale;
  const R a2n = an * an, b2n = bn * bn, c2n = cn * cn;
  const R sum = a2n + b2n;
  R disc = sum * sum - R(4) * a2n * c2n;
  if (disc < R(0)) disc = R(0);
  const R fast2n = R(0.5) * (sum + qsqrt(disc));
  const R slow2n = (fast2n > R(0)) ? (a2n * c2n) / fast2n : R(0);
  fast = scale * qsqrt(fast2n);
  slow = scale * qsqrt(slow2n);
}

// mhd_state.hpp:185-191
template <class R>
R pressure(const State<R>& u, R gamma) {
  const R kinetic = kinetic_from_momentum(u.mx, u.my, u.mz, u.rho);
  const R magnetic = half_squared_norm3(u.bx, u.by, u.bz);
  return (gamma - R(1)) * ((u.energy - kinetic) - magnetic);
}

// mhd_state.hpp:228-239
template <class R>
Prim<R> to_primitive(const State<R>& u, R gamma) {
  Prim<R> w;
  w.rho = u.rho;
  w.vx = u.mx / u.rho;
  w.vy = u.my / u.rho;
  w.vz = u.mz / u.rho;
  w.bx = u.bx;
  w.by = u.by;
  w.bz = u.bz;
  w.p = pressure(u, gamma);
  return w;
}

// mhd_state.hpp:243-256
template <class R>
State<R> to_conserved(const Prim<R>& w, R gamma) {
  State<R> u;
  u.rho = w.rho;
  u.mx = w.rho * w.vx;
  u.my = w.rho * w.vy;
  u.mz = w.rho * w.vz;
  u.bx = w.bx;
  u.by = w.by;
  u.bz = w.bz;
  const R kinetic = kinetic_from_velocity(w.rho, w.vx, w.vy, w.vz);
  const R magnetic = half_squared_norm3(w.bx, w.by, w.bz);
  u.energy = w.p / (gamma - R(1)) + kinetic + magnetic;
  return u;
}

// mhd_state.hpp:272-289 (zero background)
template <class R>
R fast_speed(const State<R>& u, int dir, R gamma) {
  const R p = pressure(u, gamma);
  R f, s, a, cn, ca;
  magnetosonic_speeds(u.rho, p, u.bx, u.by, u.bz, dir, gamma, f, s, a, cn, ca);
  return f;
}

// ---- MP limiter: mp_limiter.hpp -----------------------------------------
// mp_limiter.hpp:31-40
template <class R>
R minmod2(R a, R b) {
  if (a == R(0) || b == R(0) || ((a < R(0)) != (b < R(0)))) return R(0);
  return (qabs(a) < qabs(b)) ? a : b;
}

template <class R>
int sgn(R a) {
  return a > R(0) ? 1 : (a < R(0) ? -1 : 0);
}

// mp_limiter.hpp:44-55
template <class R>
R minmod4(R a, R b, R c, R d) {
  const int sa = sgn(a), sb = sgn(b), sc = sgn(c), sd = sgn(d);
  if (!(sa == sb && sb == sc && sc == sd) || sa == 0) return R(0);
  const R mag = qmin(qmin(qabs(a), qabs(b)), qmin(qabs(c), qabs(d)));
  return sa > 0 ? mag : -mag;
}

// mp_limiter.hpp:57-60
template <class R>
R median3(R a, R b, R c) {
  return a + minmod2(b - a, c - a);
}

// Early-accept predicate of mp_limit (mp_limiter.hpp:75-106).  True when the
// candidate is returned unchanged (no limiting).
template <class R>
bool mp_accepts(R vl, R vm1, R v0, R vp1) {
  const R alpha = R(4);
  const R d_minus = v0 - vm1;
  const R d_plus = vp1 - v0;
  const R vmp = v0 + minmod2(d_plus, alpha * d_minus);
  const R cc = vl - v0;
  const R cm = vl - vmp;
  const bool between = (cc <= R(0) && cm >= R(0)) || (cc >= R(0) && cm <= R(0));
  const R variation = qmax(qmax(qabs(d_minus), qabs(d_plus)),
                           qmax(qabs(cc), qabs(cm)));
  const bool roundoff = variation > R(0) &&
                        (qabs(cc) / variation) * (qabs(cm) / variation) <= R(1e-10);
  return between || roundoff;
}

// mp_limiter.hpp:71-148 (Cartesian face pair 1/2, 1/2, extrapolation 1/2)
template <class R>
R mp_limit(R vl, R vm2, R vm1, R v0, R vp1, R vp2, bool* fired = nullptr) {
  if (mp_accepts(vl, vm1, v0, vp1)) {
    if (fired) *fired = false;
    return vl;
  }
  if (fired) *fired = true;
  const R alpha = R(4);
  const R d_minus = v0 - vm1;
  const R dm = (vm2 - vm1) - (vm1 - v0);
  const R d0 = (vm1 - v0) - (v0 - vp1);
  const R dp = (v0 - vp1) - (vp1 - vp2);
  const R cs = qmax(qabs(dm), qmax(qabs(d0), qabs(dp)));
  R d4ph = R(0), d4mh = R(0);
  if (cs > R(0)) {
    const R dms = dm / cs, d0s = d0 / cs, dps = dp / cs;
    d4ph = cs * minmod4(R(4) * d0s - dps, R(4) * dps - d0s, d0s, dps);
    d4mh = cs * minmod4(R(4) * d0s - dms, R(4) * dms - d0s, d0s, dms);
  }
  const R v_ul = v0 + alpha * d_minus;
  const R v_av = R(0.5) * v0 + R(0.5) * vp1;
  const R v_md = v_av - R(0.5) * d4ph;
  const R v_lc = v0 + R(0.5) * d_minus + (R(4) / R(3)) * d4mh;
  const R vmin = qmax(qmin(qmin(v0, vp1), v_md), qmin(qmin(v0, v_ul), v_lc));
  const R vmax = qmin(qmax(qmax(v0, vp1), v_md), qmax(qmax(v0, v_ul), v_lc));
  return median3(vl, vmin, vmax);
}

// mp_limiter.hpp:182-191
template <class R>
R mp5_interp(R vm2, R vm1, R v0, R vp1, R vp2) {
  const R scale = qmax(qmax(qabs(vm2), qabs(vm1)),
                       qmax(qabs(v0), qmax(qabs(vp1), qabs(vp2))));
  if (scale == R(0)) return R(0);
  const R sum = R(2) * (vm2 / scale) - R(13) * (vm1 / scale) +
                R(47) * (v0 / scale) + R(27) * (vp1 / scale) -
                R(3) * (vp2 / scale);
  return (sum / R(60)) * scale;
}

// mp_limiter.hpp:196-207
template <class R>
R mp7_interp(R vm3, R vm2, R vm1, R v0, R vp1, R vp2, R vp3) {
  const R scale = qmax(qmax(qmax(qabs(vm3), qabs(vm2)), qmax(qabs(vm1), qabs(v0))),
                       qmax(qabs(vp1), qmax(qabs(vp2), qabs(vp3))));
  if (scale == R(0)) return R(0);
  const R sum = -R(3) * (vm3 / scale) + R(25) * (vm2 / scale) -
                R(101) * (vm1 / scale) + R(319) * (v0 / scale) +
                R(214) * (vp1 / scale) - R(38) * (vp2 / scale) +
                R(4) * (vp3 / scale);
  return (sum / R(420)) * scale;
}

// mp_limiter.hpp:211-224: width 5 (MP5) or 7 (MP7) window, limiter on the
// central five points.
template <class R>
R mp_reconstruct(const R* v, int width, bool* fired = nullptr) {
  if (width == 5) {
    const R vl = mp5_interp(v[0], v[1], v[2], v[3], v[4]);
    return mp_limit(vl, v[0], v[1], v[2], v[3], v[4], fired);
  }
  const R vl = mp7_interp(v[0], v[1], v[2], v[3], v[4], v[5], v[6]);
  return mp_limit(vl, v[1], v[2], v[3], v[4], v[5], fired);
}

// ---- 7-wave eigensystem: mhd_eigensystem.hpp:58-431 (B0 inactive, dir=0)
template <class R>
struct Eigen {
  R L[49];  // rows = waves
  R Rm[49]; // Rm[var*7+k] = R[var][k]
  R speeds[7];
};

template <class R>
void build_eigensystem(const State<R>& s, R gamma, Eigen<R>& e) {
  const Prim<R> w = to_primitive(s, gamma);
  const R rho = w.rho;
  const R p = (w.p > R(0)) ? w.p : R(0);
  const R sqrt_rho = qsqrt(rho);
  const R bn = w.bx, bt1 = w.by, bt2 = w.bz;
  R cf, cs, a, cax, ca;
  magnetosonic_speeds(rho, p, bn, bt1, bt2, 0, gamma, cf, cs, a, cax, ca);
  R alpha_f, alpha_s;
  {
    const R speed_scale = (cf > R(0)) ? cf : R(1);
    const R cfn = cf / speed_scale, csn = cs / speed_scale, an = a / speed_scale;
    const R denom = cfn * cfn - csn * csn;
    const R eps = R(64.0 * kEps);
    if (denom <= eps * (cfn * cfn + csn * csn)) {
      alpha_f = R(1) / qsqrt(R(2));
      alpha_s = R(1) / qsqrt(R(2));
    } else {
      R af2 = (an * an - csn * csn) / denom;
      R as2 = (cfn * cfn - an * an) / denom;
      if (af2 < R(0)) af2 = R(0);
      if (as2 < R(0)) as2 = R(0);
      alpha_f = qsqrt(af2);
      alpha_s = qsqrt(as2);
    }
  }
  R beta1, beta2;
  {
    const R bt = scaled_norm3(bt1, bt2, R(0));
    const R bt_speed = bt / sqrt_rho;
    const R field_scale = (a > ca) ? a : ca;
    const R eps = R(64.0 * kEps);
    if (bt == R(0) || bt_speed <= eps * (field_scale + R(kTiny))) {
      beta1 = R(1) / qsqrt(R(2));
      beta2 = R(1) / qsqrt(R(2));
    } else {
      beta1 = bt1 / bt;
      beta2 = bt2 / bt;
    }
  }
  const R sbn = (bn >= R(0)) ? R(1) : R(-1);
  const R vn = w.vx, vt1 = w.vy, vt2 = w.vz;
  e.speeds[0] = vn - cf;
  e.speeds[1] = vn - cax;
  e.speeds[2] = vn - cs;
  e.speeds[3] = vn;
  e.speeds[4] = vn + cs;
  e.speeds[5] = vn + cax;
  e.speeds[6] = vn + cf;

  const R qf = cf * alpha_f * sbn;
  const R qs = cs * alpha_s * sbn;
  const R Af = a * alpha_f * sqrt_rho;
  const R As = a * alpha_s * sqrt_rho;
  const R inv_a2 = (a > R(0)) ? (R(1) / a) / a : R(0);
  const R Nf = R(0.5) * inv_a2;
  const R rho_a2 = gamma * p;
  const R s2 = R(1) / qsqrt(R(2));

  R Rp[7][7], Lp[7][7];
  for (int k = 0; k < 7; ++k)
    for (int v = 0; v < 7; ++v) { Rp[k][v] = R(0); Lp[k][v] = R(0); }
  // mhd_eigensystem.hpp:176-259
  Rp[0][0] = rho * alpha_f; Rp[0][1] = -alpha_f * cf; Rp[0][2] = qs * beta1;
  Rp[0][3] = qs * beta2;    Rp[0][4] = alpha_f * rho_a2;
  Rp[0][5] = As * beta1;    Rp[0][6] = As * beta2;
  Rp[6][0] = rho * alpha_f; Rp[6][1] = alpha_f * cf;  Rp[6][2] = -qs * beta1;
  Rp[6][3] = -qs * beta2;   Rp[6][4] = alpha_f * rho_a2;
  Rp[6][5] = As * beta1;    Rp[6][6] = As * beta2;
  Rp[1][2] = -beta2 * s2;   Rp[1][3] = beta1 * s2;
  Rp[1][5] = -sbn * beta2 * s2 * sqrt_rho;
  Rp[1][6] = sbn * beta1 * s2 * sqrt_rho;
  Rp[5][2] = -beta2 * s2;   Rp[5][3] = beta1 * s2;
  Rp[5][5] = sbn * beta2 * s2 * sqrt_rho;
  Rp[5][6] = -sbn * beta1 * s2 * sqrt_rho;
  Rp[2][0] = rho * alpha_s; Rp[2][1] = -alpha_s * cs; Rp[2][2] = -qf * beta1;
  Rp[2][3] = -qf * beta2;   Rp[2][4] = alpha_s * rho_a2;
  Rp[2][5] = -Af * beta1;   Rp[2][6] = -Af * beta2;
  Rp[4][0] = rho * alpha_s; Rp[4][1] = alpha_s * cs;  Rp[4][2] = qf * beta1;
  Rp[4][3] = qf * beta2;    Rp[4][4] = alpha_s * rho_a2;
  Rp[4][5] = -Af * beta1;   Rp[4][6] = -Af * beta2;
  Rp[3][0] = R(1);
  // mhd_eigensystem.hpp:263-320
  Lp[0][1] = -Nf * alpha_f * cf; Lp[0][2] = Nf * qs * beta1;
  Lp[0][3] = Nf * qs * beta2;    Lp[0][4] = Nf * alpha_f / rho;
  Lp[0][5] = Nf * As * beta1 / rho; Lp[0][6] = Nf * As * beta2 / rho;
  Lp[6][1] = Nf * alpha_f * cf;  Lp[6][2] = -Nf * qs * beta1;
  Lp[6][3] = -Nf * qs * beta2;   Lp[6][4] = Nf * alpha_f / rho;
  Lp[6][5] = Nf * As * beta1 / rho; Lp[6][6] = Nf * As * beta2 / rho;
  Lp[1][2] = -beta2 * s2; Lp[1][3] = beta1 * s2;
  Lp[1][5] = -sbn * beta2 * s2 / sqrt_rho; Lp[1][6] = sbn * beta1 * s2 / sqrt_rho;
  Lp[5][2] = -beta2 * s2; Lp[5][3] = beta1 * s2;
  Lp[5][5] = sbn * beta2 * s2 / sqrt_rho; Lp[5][6] = -sbn * beta1 * s2 / sqrt_rho;
  Lp[2][1] = -Nf * alpha_s * cs; Lp[2][2] = -Nf * qf * beta1;
  Lp[2][3] = -Nf * qf * beta2;   Lp[2][4] = Nf * alpha_s / rho;
  Lp[2][5] = -Nf * Af * beta1 / rho; Lp[2][6] = -Nf * Af * beta2 / rho;
  Lp[4][1] = Nf * alpha_s * cs;  Lp[4][2] = Nf * qf * beta1;
  Lp[4][3] = Nf * qf * beta2;    Lp[4][4] = Nf * alpha_s / rho;
  Lp[4][5] = -Nf * Af * beta1 / rho; Lp[4][6] = -Nf * Af * beta2 / rho;
  Lp[3][0] = R(1); Lp[3][4] = -inv_a2;

  // mhd_eigensystem.hpp:332-388: M = dU/dW, Minv = dW/dU (B0 inactive).
  const R gm1 = gamma - R(1);
  const R half_v2 = half_squared_norm3(vn, vt1, vt2);
  R M[7][7], Mi[7][7];
  for (int r = 0; r < 7; ++r)
    for (int c = 0; c < 7; ++c) { M[r][c] = R(0); Mi[r][c] = R(0); }
  M[0][0] = R(1);
  M[1][0] = vn;  M[1][1] = rho;
  M[2][0] = vt1; M[2][2] = rho;
  M[3][0] = vt2; M[3][3] = rho;
  M[4][0] = half_v2; M[4][1] = rho * vn; M[4][2] = rho * vt1; M[4][3] = rho * vt2;
  M[4][4] = R(1) / gm1; M[4][5] = bt1; M[4][6] = bt2;
  M[5][5] = R(1); M[6][6] = R(1);
  const R inv_rho = R(1) / rho;
  Mi[0][0] = R(1);
  Mi[1][0] = -vn * inv_rho;  Mi[1][1] = inv_rho;
  Mi[2][0] = -vt1 * inv_rho; Mi[2][2] = inv_rho;
  Mi[3][0] = -vt2 * inv_rho; Mi[3][3] = inv_rho;
  Mi[4][0] = gm1 * half_v2; Mi[4][1] = -gm1 * vn; Mi[4][2] = -gm1 * vt1;
  Mi[4][3] = -gm1 * vt2; Mi[4][4] = gm1; Mi[4][5] = -gm1 * bt1; Mi[4][6] = -gm1 * bt2;
  Mi[5][5] = R(1); Mi[6][6] = R(1);
  // mhd_eigensystem.hpp:392-405 (dense products as written by the reference)
  for (int k = 0; k < 7; ++k) {
    for (int v = 0; v < 7; ++v) {
      R racc = R(0), lacc = R(0);
      for (int j = 0; j < 7; ++j) {
        racc = racc + M[v][j] * Rp[k][j];
        lacc = lacc + Lp[k][j] * Mi[j][v];
      }
      e.Rm[v * 7 + k] = racc;
      e.L[k * 7 + v] = lacc;
    }
  }
  // mhd_eigensystem.hpp:416-430: biorthogonality check, identity fallback.
  bool usable = true;
  for (int i = 0; i < 7 && usable; ++i) {
    for (int j = 0; j < 7; ++j) {
      R dot = R(0);
      for (int k = 0; k < 7; ++k) dot = dot + e.L[i * 7 + k] * e.Rm[k * 7 + j];
      const R expected = (i == j) ? R(1) : R(0);
      if (!qfinite(dot) || qabs(dot - expected) > R(1024.0 * kEps)) {
        usable = false;
        break;
      }
    }
  }
  if (!usable) {
    for (int i = 0; i < 7; ++i)
      for (int j = 0; j < 7; ++j) {
        const R v = (i == j) ? R(1) : R(0);
        e.L[i * 7 + j] = v;
        e.Rm[i * 7 + j] = v;
      }
  }
}

// ---- HLLD core: hlld_core.hpp ---------------------------------------------
template <class R>
struct Flux {
  R rho, mx, my, mz, energy, bx, by, bz;
};

// hlld_core.hpp:123-153
template <class R>
Flux<R> physical_flux_x(const State<R>& u, R gamma) {
  const R vx = u.mx / u.rho, vy = u.my / u.rho, vz = u.mz / u.rho;
  const R p = pressure(u, gamma);
  const R half_bn2 = half_squared_norm3(u.bx, R(0), R(0));
  const R half_bt2 = half_squared_norm3(R(0), u.by, u.bz);
  Flux<R> f;
  f.rho = u.mx;
  {
    const R t[5] = {u.mx * vx, p * R(1), u.by * (R(0.5) * u.by), u.bz * (R(0.5) * u.bz),
                    u.bx * (R(-0.5) * u.bx)};
    f.mx = crsum(t, 5);
  }
  f.my = u.mx * vy + u.bx * (-u.by);
  f.mz = u.mx * vz + u.bx * (-u.bz);
  const R normal_enthalpy = ((u.energy - half_bn2) + p) + half_bt2;
  const R tvb = vy * u.by + vz * u.bz;
  f.energy = vx * normal_enthalpy + u.bx * (-tvb);
  f.bx = R(0);
  f.by = u.by * vx + u.bx * (-vy);
  f.bz = u.bz * vx + u.bx * (-vz);
  return f;
}

// hlld_core.hpp:157-192
template <class R>
Flux<R> hll_flux_x(const State<R>& L, const State<R>& Rs, R sl, R sr, R gamma) {
  const Flux<R> fl = physical_flux_x(L, gamma);
  const Flux<R> fr = physical_flux_x(Rs, gamma);
  if (sl >= R(0)) return fl;
  if (sr <= R(0)) return fr;
  const R speed_scale = qmax(qabs(sl), qabs(sr));
  if (!(speed_scale > R(0)) || !qfinite(speed_scale)) return fl;
  const R sln = sl / speed_scale, srn = sr / speed_scale;
  const R denom = srn - sln;
  if (!(denom > R(0)) || !qfinite(denom)) return fl;
  const R wl = srn / denom, wr = -sln / denom;
  const R dis = speed_scale * (sln * srn / denom);
  Flux<R> f;
  f.rho = crsum3(wl * fl.rho, wr * fr.rho, dis * (Rs.rho - L.rho));
  f.mx = crsum3(wl * fl.mx, wr * fr.mx, dis * (Rs.mx - L.mx));
  f.my = crsum3(wl * fl.my, wr * fr.my, dis * (Rs.my - L.my));
  f.mz = crsum3(wl * fl.mz, wr * fr.mz, dis * (Rs.mz - L.mz));
  f.energy = crsum3(wl * fl.energy, wr * fr.energy, dis * (Rs.energy - L.energy));
  f.bx = R(0);
  f.by = crsum3(wl * fl.by, wr * fr.by, dis * (Rs.by - L.by));
  f.bz = crsum3(wl * fl.bz, wr * fr.bz, dis * (Rs.bz - L.bz));
  return f;
}

// hlld_core.hpp:200-210
template <class R>
Flux<R> lax_friedrichs_flux_x(const State<R>& L, const State<R>& Rs, R gamma) {
  const R vxL = L.mx / L.rho, vxR = Rs.mx / Rs.rho;
  const R aL = qabs(vxL) + fast_speed(L, 0, gamma);
  const R aR = qabs(vxR) + fast_speed(Rs, 0, gamma);
  const R alpha = (aL > aR) ? aL : aR;
  return hll_flux_x(L, Rs, -alpha, alpha, gamma);
}

template <class R>
bool same_state(const State<R>& a, const State<R>& b) {
  return a.rho == b.rho && a.mx == b.mx && a.my == b.my && a.mz == b.mz &&
         a.energy == b.energy && a.bx == b.bx && a.by == b.by && a.bz == b.bz;
}

template <class R>
bool flux_finite(const Flux<R>& f) {
  return qfinite(f.rho) && qfinite(f.mx) && qfinite(f.my) && qfinite(f.mz) &&
         qfinite(f.energy) && qfinite(f.by) && qfinite(f.bz);
}

// hlld_core.hpp:213-457
template <class R>
Flux<R> hlld_flux_x(const State<R>& Lin, const State<R>& Rin, R gamma) {
  const R rel_tol = R(64.0 * kEps);
  auto resolved = [&](R value, R scale) {
    return qfinite(value) && qabs(value) > rel_tol * (scale + R(kTiny));
  };
  if (same_state(Lin, Rin)) return physical_flux_x(Lin, gamma);

  const R bn = R(0.5) * Lin.bx + R(0.5) * Rin.bx;
  State<R> L = Lin, Rs = Rin;
  const R half_bn2 = half_squared_norm3(bn, R(0), R(0));
  L.energy = (L.energy - half_squared_norm3(L.bx, R(0), R(0))) + half_bn2;
  Rs.energy = (Rs.energy - half_squared_norm3(Rs.bx, R(0), R(0))) + half_bn2;
  L.bx = bn;
  Rs.bx = bn;
  const bool bn2_ok = qval(half_bn2) <= 0.5 * std::numeric_limits<double>::max();
  const R bn2 = bn2_ok ? R(2) * half_bn2 : R(0);

  const R irl = R(1) / L.rho, irr = R(1) / Rs.rho;
  const R vxL = L.mx * irl, vyL = L.my * irl, vzL = L.mz * irl;
  const R vxR = Rs.mx * irr, vyR = Rs.my * irr, vzR = Rs.mz * irr;
  const R pL = pressure(L, gamma), pR = pressure(Rs, gamma);
  const R ptL = pL + half_squared_norm3(L.bx, L.by, L.bz);
  const R ptR = pR + half_squared_norm3(Rs.bx, Rs.by, Rs.bz);
  const R cfL = fast_speed(L, 0, gamma), cfR = fast_speed(Rs, 0, gamma);
  const R cfmax = (cfL > cfR) ? cfL : cfR;
  const R sl = ((vxL < vxR) ? vxL : vxR) - cfmax;
  const R sr = ((vxL > vxR) ? vxL : vxR) + cfmax;
  if (sl >= R(0)) return physical_flux_x(L, gamma);
  if (sr <= R(0)) return physical_flux_x(Rs, gamma);
  if (!bn2_ok || !qfinite(ptL) || !qfinite(ptR)) return hll_flux_x(L, Rs, sl, sr, gamma);

  const R denomM = (sr - vxR) * Rs.rho - (sl - vxL) * L.rho;
  const R denomM_scale = qabs((sr - vxR) * Rs.rho) + qabs((sl - vxL) * L.rho);
  if (!resolved(denomM, denomM_scale)) return hll_flux_x(L, Rs, sl, sr, gamma);
  const R sm = ((sr - vxR) * Rs.rho * vxR - (sl - vxL) * L.rho * vxL - ptR + ptL) / denomM;
  if (!qfinite(sm)) return hll_flux_x(L, Rs, sl, sr, gamma);
  const R pt_star = ((sr - vxR) * Rs.rho * ptL - (sl - vxL) * L.rho * ptR +
                     L.rho * Rs.rho * (sr - vxR) * (sl - vxL) * (vxR - vxL)) / denomM;
  if (!qfinite(pt_star)) return hll_flux_x(L, Rs, sl, sr, gamma);
  const R dLs = sl - sm, dRs = sr - sm;
  const R wave_scale = qabs(sl) + qabs(sr) + qabs(sm);
  if (!resolved(dLs, wave_scale) || !resolved(dRs, wave_scale))
    return hll_flux_x(L, Rs, sl, sr, gamma);
  const R rhoLs = L.rho * (sl - vxL) / dLs;
  const R rhoRs = Rs.rho * (sr - vxR) / dRs;
  if (!(rhoLs > R(0)) || !(rhoRs > R(0))) return hll_flux_x(L, Rs, sl, sr, gamma);

  struct Star {
    State<R> u;
    R vy, vz, by, bz;
    bool ok;
  };
  auto star_state = [&](const State<R>& U, R s, R vx, R vy, R vz, R pt, R rhos) {
    Star out;
    out.ok = true;
    const R smv = s - vx;
    const R denom = U.rho * smv * (s - sm) - bn2;
    const R denom_scale = qabs(U.rho * smv * (s - sm)) + bn2;
    if (!resolved(denom, denom_scale)) {
      out.ok = false;
      return out;
    }
    const R inv_denom = R(1) / denom;
    const R fac = bn * (sm - vx) * inv_denom;
    const R vys = vy - U.by * fac;
    const R vzs = vz - U.bz * fac;
    const R bcoef = (U.rho * smv * smv - bn2) * inv_denom;
    const R bys = U.by * bcoef;
    const R bzs = U.bz * bcoef;
    State<R> us;
    us.rho = rhos;
    us.bx = bn;
    us.mx = us.rho * sm;
    us.my = us.rho * vys;
    us.mz = us.rho * vzs;
    us.by = bys;
    us.bz = bzs;
    const R vdotb = crsum3(vx * U.bx, vy * U.by, vz * U.bz);
    const R vdotb_s = crsum3(sm * bn, vys * bys, vzs * bzs);
    us.energy = (smv * U.energy - pt * vx + pt_star * sm + bn * (vdotb - vdotb_s)) / (s - sm);
    out.u = us;
    out.vy = vys;
    out.vz = vzs;
    out.by = bys;
    out.bz = bzs;
    return out;
  };
  const Star sL = star_state(L, sl, vxL, vyL, vzL, ptL, rhoLs);
  const Star sR = star_state(Rs, sr, vxR, vyR, vzR, ptR, rhoRs);
  if (!sL.ok || !sR.ok) return hll_flux_x(L, Rs, sl, sr, gamma);
  const Flux<R> fl = physical_flux_x(L, gamma);
  const Flux<R> fr = physical_flux_x(Rs, gamma);
  auto from_star = [&](const Flux<R>& fU, const State<R>& U, const State<R>& us, R s) {
    Flux<R> f;
    f.rho = fU.rho + s * (us.rho - U.rho);
    f.mx = fU.mx + s * (us.mx - U.mx);
    f.my = fU.my + s * (us.my - U.my);
    f.mz = fU.mz + s * (us.mz - U.mz);
    f.energy = fU.energy + s * (us.energy - U.energy);
    f.bx = R(0);
    f.by = fU.by + s * (us.by - U.by);
    f.bz = fU.bz + s * (us.bz - U.bz);
    return f;
  };
  const R srLs = qsqrt(rhoLs), srRs = qsqrt(rhoRs);
  const R saL = sm - qabs(bn) / srLs;
  const R saR = sm + qabs(bn) / srRs;
  const bool bn_negl = bn2 <= rel_tol * (qabs(pt_star) + qabs(ptL) + qabs(ptR) + R(kTiny));
  if (bn_negl) {
    Flux<R> f = (sl <= R(0) && R(0) <= sm) ? from_star(fl, L, sL.u, sl)
                                           : from_star(fr, Rs, sR.u, sr);
    if (!qfinite(f.rho) || !qfinite(f.energy)) return hll_flux_x(L, Rs, sl, sr, gamma);
    return f;
  }
  const R inv_sum = R(1) / (srLs + srRs);
  const R sg = (bn >= R(0)) ? R(1) : R(-1);
  const R vyss = (srLs * sL.vy + srRs * sR.vy + (sR.by - sL.by) * sg) * inv_sum;
  const R vzss = (srLs * sL.vz + srRs * sR.vz + (sR.bz - sL.bz) * sg) * inv_sum;
  const R byss = (srLs * sR.by + srRs * sL.by + srLs * srRs * (sR.vy - sL.vy) * sg) * inv_sum;
  const R bzss = (srLs * sR.bz + srRs * sL.bz + srLs * srRs * (sR.vz - sL.vz) * sg) * inv_sum;
  auto double_star = [&](const Star& s, R sqrt_rhos, R side) {
    State<R> u;
    u.rho = s.u.rho;
    u.bx = bn;
    u.mx = u.rho * sm;
    u.my = u.rho * vyss;
    u.mz = u.rho * vzss;
    u.by = byss;
    u.bz = bzss;
    const R vb_ss = crsum3(sm * bn, vyss * byss, vzss * bzss);
    const R vb_s = crsum3(sm * bn, s.vy * s.by, s.vz * s.bz);
    u.energy = s.u.energy + side * sqrt_rhos * sg * (vb_s - vb_ss);
    return u;
  };
  const State<R> ussL = double_star(sL, srLs, R(-1));
  const State<R> ussR = double_star(sR, srRs, R(1));
  Flux<R> f;
  if (R(0) <= saL) {
    f = from_star(fl, L, sL.u, sl);
  } else if (R(0) <= sm) {
    const State<R>& a = sL.u;
    f.rho = fl.rho + saL * (ussL.rho - a.rho) + sl * (a.rho - L.rho);
    f.mx = fl.mx + saL * (ussL.mx - a.mx) + sl * (a.mx - L.mx);
    f.my = fl.my + saL * (ussL.my - a.my) + sl * (a.my - L.my);
    f.mz = fl.mz + saL * (ussL.mz - a.mz) + sl * (a.mz - L.mz);
    f.energy = fl.energy + saL * (ussL.energy - a.energy) + sl * (a.energy - L.energy);
    f.bx = R(0);
    f.by = fl.by + saL * (ussL.by - a.by) + sl * (a.by - L.by);
    f.bz = fl.bz + saL * (ussL.bz - a.bz) + sl * (a.bz - L.bz);
  } else if (R(0) <= saR) {
    const State<R>& a = sR.u;
    f.rho = fr.rho + saR * (ussR.rho - a.rho) + sr * (a.rho - Rs.rho);
    f.mx = fr.mx + saR * (ussR.mx - a.mx) + sr * (a.mx - Rs.mx);
    f.my = fr.my + saR * (ussR.my - a.my) + sr * (a.my - Rs.my);
    f.mz = fr.mz + saR * (ussR.mz - a.mz) + sr * (a.mz - Rs.mz);
    f.energy = fr.energy + saR * (ussR.energy - a.energy) + sr * (a.energy - Rs.energy);
    f.bx = R(0);
    f.by = fr.by + saR * (ussR.by - a.by) + sr * (a.by - Rs.by);
    f.bz = fr.bz + saR * (ussR.bz - a.bz) + sr * (a.bz - Rs.bz);
  } else {
    f = from_star(fr, Rs, sR.u, sr);
  }
  if (!flux_finite(f)) return hll_flux_x(L, Rs, sl, sr, gamma);
  return f;
}

// Transverse quadrature tables: finite_volume_quadrature.hpp:12-48.
inline constexpr double kGauss3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
inline constexpr double kGauss4[4] = {0.173927422568726925, 0.326072577431273103,
                                      0.326072577431273103, 0.173927422568726925};
inline constexpr double kPoint5[3][5] = {
    {-0.0392523473402346598, 0.312987195324173573, 0.910833333333333384,
     -0.216320528657506839, 0.0317523473402346601},
    {0.00468749999999999983, -0.0604166666666666671, 1.11145833333333344,
     -0.0604166666666666671, 0.00468749999999999983},
    {0.0317523473402346601, -0.216320528657506839, 0.910833333333333384,
     0.312987195324173573, -0.0392523473402346598}};
inline constexpr double kPoint7[4][7] = {
    {0.00860109764472105458, -0.0796691475531970394, 0.415576982717296983,
     0.849155569794037945, -0.245805403605616202, 0.0591434746546156687,
     -0.0070025736518584264},
    {0.00327670662777140203, -0.0266359260617751309, 0.0928282644451935562,
     1.08046056237311472, -0.183384586025290314, 0.0375843394851378479,
     -0.00412936084415200903},
    {-0.00412936084415200903, 0.0375843394851378479, -0.183384586025290314,
     1.08046056237311472, 0.0928282644451935562, -0.0266359260617751309,
     0.00327670662777140203},
    {-0.0070025736518584264, 0.0591434746546156687, -0.245805403605616202,
     0.849155569794037945, 0.415576982717296983, -0.0796691475531970394,
     0.00860109764472105458}};

// finite_volume_quadrature.hpp:55-68: weighted sum with the exact constant
// shortcut (all samples equal to the centre one -> return it unchanged).
template <class R>
R weighted_value(const double* w, const R* s, int count) {
  const R ref = s[count / 2];
  bool constant = true;
  for (int q = 0; q < count; ++q) constant = constant && (s[q] == ref);
  if (constant) return ref;
  R t[8];
  for (int q = 0; q < count; ++q) t[q] = R(w[q]) * s[q];
  return crsum(t, count);
}

}  // namespace qoracle
