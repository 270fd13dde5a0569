// Device numerics of the 2-D ideal-MHD step (sm_100a, FP64).
//
// Pointwise formulas follow the reference's numerics headers formula by
// formula (cited per function, paths relative to the quasar tree) so that the
// result matches its own path to rounding.  The reference evaluates many sums
// through exact-expansion arithmetic (numerics/scaled_arithmetic.hpp).  Here
// ordinary FP64 (with FMA contraction) is used everywhere except at the sites
// where the exact sum creates an exact invariance the algorithm branches on:
// collocating a constant face field returns the constant, and replacing the
// normal field by an equal value leaves the energy bit-identical.  Those sites
// use compensated sums built from non-contracting IEEE intrinsics.
#pragma once

#include <cstdint>

namespace qb {

struct St {
  double rho, mx, my, mz, E, bx, by, bz;
};
struct Pr {
  double rho, vx, vy, vz, p, bx, by, bz;
};
struct Fx {
  double rho, mx, my, mz, E, bx, by, bz;
};

__host__ __device__ inline double comp(const St& s, int c) {
  switch (c) {
    case 0: return s.rho;
    case 1: return s.mx;
    case 2: return s.my;
    case 3: return s.mz;
    case 4: return s.E;
    case 5: return s.bx;
    case 6: return s.by;
    default: return s.bz;
  }
}

constexpr double kEps = 2.220446049250313080847e-16;
constexpr double kTiny = 2.2250738585072014e-308;
constexpr double kInf = __builtin_huge_val();

// ---- compensated sums (never contracted) ---------------------------------
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dadd_rn(s, -a);
  e = __dadd_rn(__dadd_rn(a, -__dadd_rn(s, -bb)), __dadd_rn(b, -bb));
}
// Correctly rounded (up to rare ties) a+b+c of already rounded terms.
__device__ __forceinline__ double crsum3(double a, double b, double c) {
  double s, e1, e2;
  two_sum(a, b, s, e1);
  two_sum(s, c, s, e2);
  return __dadd_rn(s, __dadd_rn(e1, e2));
}
// Sum of exact products w[k]*x[k], rounded once (Dot2).
template <int N>
__device__ __forceinline__ double exact_dot(const double* w, const double* x) {
  double s = __dmul_rn(w[0], x[0]);
  double c = fma(w[0], x[0], -s);
#pragma unroll
  for (int k = 1; k < N; ++k) {
    const double p = __dmul_rn(w[k], x[k]);
    const double pe = fma(w[k], x[k], -p);
    double e;
    two_sum(s, p, s, e);
    c = __dadd_rn(c, __dadd_rn(e, pe));
  }
  return __dadd_rn(s, c);
}

// ---- division by a cell size ----------------------------------------------
// Reciprocal of h when h is a power of two whose reciprocal is a normal
// number (then it is exact), else 0.
__device__ __forceinline__ double pow2_recip(double h) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(h);
  const unsigned e = unsigned(b >> 52) & 0x7ffu;
  const bool pow2 = (b & 0x000fffffffffffffull) == 0ull && e >= 2u && e <= 2044u;
  return pow2 ? 1.0 / h : 0.0;
}
// x / h, formed as x * (1/h) where pow2_recip gave the exact reciprocal rh:
// both are the correctly rounded value of the same real number, so the bits
// are those of the division (every grid whose side is a power-of-two number
// of cells on a unit box takes the multiplication).
__device__ __forceinline__ double div_by(double x, double h, double rh) {
  return rh != 0.0 ? __dmul_rn(x, rh) : __ddiv_rn(x, h);
}

// ---- EOS helpers: numerics/mhd_state.hpp ---------------------------------
// Evaluated without FMA contraction, in the reference's operation order: at a
// degenerate wave fan (zero transverse field) the eigenvector weights are
// square roots of rounding-level differences of these quantities, so their
// bits decide the branch.
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double sq3(double x, double y, double z) {
  return add(add(mul(x, x), mul(y, y)), mul(z, z));
}
// mhd_state.hpp:92-100
__device__ __forceinline__ double scaled_norm3(double x, double y, double z) {
  const double s = fmax(fabs(x), fmax(fabs(y), fabs(z)));
  if (s == 0.0) return 0.0;
  return mul(s, sqrt(sq3(x / s, y / s, z / s)));
}
// mhd_state.hpp:105-114
__device__ __forceinline__ double half_sq3(double x, double y, double z) {
  const double s = fmax(fabs(x), fmax(fabs(y), fabs(z)));
  if (s == 0.0) return 0.0;
  return mul(mul(0.5, s), mul(s, sq3(x / s, y / s, z / s)));
}
// mhd_state.hpp:118-128
__device__ __forceinline__ double kin_mom(double mx, double my, double mz, double rho) {
  const double s = fmax(fabs(mx), fmax(fabs(my), fabs(mz)));
  if (s == 0.0) return 0.0;
  const double q = s / sqrt(rho);
  return mul(mul(0.5, q), mul(q, sq3(mx / s, my / s, mz / s)));
}
// mhd_state.hpp:131-141
__device__ __forceinline__ double kin_vel(double rho, double vx, double vy, double vz) {
  const double s = fmax(fabs(vx), fmax(fabs(vy), fabs(vz)));
  if (s == 0.0) return 0.0;
  const double q = mul(sqrt(rho), s);
  return mul(mul(0.5, q), mul(q, sq3(vx / s, vy / s, vz / s)));
}
// mhd_state.hpp:148-182, normal Alfven component along x
__device__ __forceinline__ void magnetosonic(double rho, double p, double bn, double bt1,
                                             double bt2, double gamma, double& fast,
                                             double& slow, double& sound, double& can,
                                             double& ca) {
  const double sr = sqrt(rho);
  sound = (p > 0.0 && gamma > 0.0) ? mul(sqrt(gamma), sqrt(p) / sr) : 0.0;
  const double ax = bn / sr, ay = bt1 / sr, az = bt2 / sr;
  ca = scaled_norm3(ax, ay, az);
  can = fabs(ax);
  const double scale = fmax(sound, ca);
  if (!(scale > 0.0)) {
    fast = 0.0;
    slow = 0.0;
    return;
  }
  const double an = sound / scale, bnn = ca / scale, cn = can / scale;
  const double a2 = mul(an, an), b2 = mul(bnn, bnn), c2 = mul(cn, cn);
  const double sum = add(a2, b2);
  double disc = sub(mul(sum, sum), mul(mul(4.0, a2), c2));
  if (disc < 0.0) disc = 0.0;
  const double f2 = mul(0.5, add(sum, sqrt(disc)));
  const double s2 = (f2 > 0.0) ? mul(a2, c2) / f2 : 0.0;
  fast = mul(scale, sqrt(f2));
  slow = mul(scale, sqrt(s2));
}
// mhd_state.hpp:185-191
__device__ __forceinline__ double pressure(const St& u, double gamma) {
  const double k = kin_mom(u.mx, u.my, u.mz, u.rho);
  const double m = half_sq3(u.bx, u.by, u.bz);
  return mul(sub(gamma, 1.0), sub(sub(u.E, k), m));
}
// Plain-arithmetic EOS for the places whose result depends continuously on
// rounding (Riemann solver, CFL speeds, admissibility tests): one reciprocal
// of rho instead of the reference's component-scaled forms, which only guard
// binary64 overflow for |state| near 1e154 (outside every configuration here).
__device__ __forceinline__ double pressure_f(const St& u, double gamma, double ir) {
  const double k = 0.5 * ((u.mx * u.mx + u.my * u.my + u.mz * u.mz) * ir);
  const double m = 0.5 * (u.bx * u.bx + u.by * u.by + u.bz * u.bz);
  return (gamma - 1.0) * ((u.E - k) - m);
}
// fast magnetosonic speed normal to x from p and 1/rho (mhd_state.hpp:148-182);
// discriminant as (a^2 - b^2)^2 + 4 a^2 b_t^2, free of cancellation
__device__ __forceinline__ double fast_x_f(const St& u, double p, double ir, double gamma) {
  const double a2 = p > 0.0 ? gamma * p * ir : 0.0;
  const double bn2 = u.bx * u.bx * ir;
  const double bt2 = (u.by * u.by + u.bz * u.bz) * ir;
  const double d = a2 - (bn2 + bt2);
  const double disc = d * d + 4.0 * a2 * bt2;
  return sqrt(0.5 * ((a2 + bn2 + bt2) + sqrt(disc)));
}

__device__ __forceinline__ Pr to_prim(const St& u, double gamma) {
  Pr w;
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
__device__ __forceinline__ St to_cons(const Pr& w, double gamma) {
  St u;
  u.rho = w.rho;
  u.mx = w.rho * w.vx;
  u.my = w.rho * w.vy;
  u.mz = w.rho * w.vz;
  u.bx = w.bx;
  u.by = w.by;
  u.bz = w.bz;
  u.E = w.p / (gamma - 1.0) + kin_vel(w.rho, w.vx, w.vy, w.vz) + half_sq3(w.bx, w.by, w.bz);
  return u;
}
// mhd_state.hpp:272-289 (x-normal)
__device__ __forceinline__ double fast_x(const St& u, double gamma) {
  double f, s, a, cn, ca;
  magnetosonic(u.rho, pressure(u, gamma), u.bx, u.by, u.bz, gamma, f, s, a, cn, ca);
  return f;
}

// x<->y swap of the in-plane momentum and field (mhd_reconstruct.hip:167-176,
// hlld_core.hpp:45-61).
__device__ __forceinline__ St swap_xy(const St& v) {
  St r = v;
  r.mx = v.my;
  r.my = v.mx;
  r.bx = v.by;
  r.by = v.bx;
  return r;
}

// Finite, rho>0, finite velocity, p>0 (mhd_reconstruct.hip:414-427).
__device__ __forceinline__ bool recon_admissible(const St& s, double gamma) {
  if (!(isfinite(s.rho) && s.rho > 0.0)) return false;
  const double ir = 1.0 / s.rho;
  const double p = pressure_f(s, gamma, ir);
  if (!(isfinite(s.mx * ir) && isfinite(s.my * ir) && isfinite(s.mz * ir) && isfinite(p) &&
        p > 0.0))
    return false;
  return isfinite(s.mx) && isfinite(s.my) && isfinite(s.mz) && isfinite(s.E) &&
         isfinite(s.bx) && isfinite(s.by) && isfinite(s.bz);
}
// mhd_face_quadrature.hpp:68-76, with 1/rho supplied.  Every component
// enters the pressure, so with rho finite and positive "p finite and
// positive" already fails for any non-finite component (an infinite momentum
// or field drives p to -inf, an infinite energy to +/-inf, a NaN to NaN): the
// reference's per-component finiteness tests are implied and not repeated,
// the decision is the same.
__device__ __forceinline__ bool point_admissible_ir(const St& s, double gamma, double ir) {
  if (!(isfinite(s.rho) && s.rho > 0.0)) return false;
  const double p = pressure_f(s, gamma, ir);
  return isfinite(p) && p > 0.0;
}
__device__ __forceinline__ bool point_admissible(const St& s, double gamma) {
  return point_admissible_ir(s, gamma, 1.0 / s.rho);
}

// ---- MP limiter: numerics/mp_limiter.hpp ---------------------------------
__device__ __forceinline__ double minmod2(double a, double b) {
  if (a == 0.0 || b == 0.0 || ((a < 0.0) != (b < 0.0))) return 0.0;
  return (fabs(a) < fabs(b)) ? a : b;
}
__device__ __forceinline__ int sgn(double a) { return a > 0.0 ? 1 : (a < 0.0 ? -1 : 0); }
__device__ __forceinline__ double minmod4(double a, double b, double c, double d) {
  const int sa = sgn(a);
  if (!(sa == sgn(b) && sa == sgn(c) && sa == sgn(d)) || sa == 0) return 0.0;
  const double m = fmin(fmin(fabs(a), fabs(b)), fmin(fabs(c), fabs(d)));
  return sa > 0 ? m : -m;
}
// mp_limiter.hpp:71-148.  `fired` is set when the candidate was changed.
// The normalisations by the local variation and the curvature scale use one
// reciprocal each instead of a division per term (rounding-level difference).
// Not inlined: the warp-cooperative reconstruction calls it four times per
// round, and one shared body instead of four inlined copies relieves its
// instruction-fetch stalls (reconstruction 37.0 -> 35.5 ms per rotor 4096^2
// MP7 step, 12.6 -> 11.3 on Orszag-Tang 2048^2 MP7; the state bit-identical).
__device__ __noinline__ double mp_limit(double vl, double vm2, double vm1, double v0,
                                           double vp1, double vp2, bool& fired) {
  const double dmn = v0 - vm1;
  const double dpl = vp1 - v0;
  const double vmp = v0 + minmod2(dpl, 4.0 * dmn);
  const double cc = vl - v0, cm = vl - vmp;
  const bool between = (cc <= 0.0 && cm >= 0.0) || (cc >= 0.0 && cm <= 0.0);
  const double var = fmax(fmax(fabs(dmn), fabs(dpl)), fmax(fabs(cc), fabs(cm)));
  bool roundoff = false;
  if (!between && var > 0.0) {
    const double iv = 1.0 / var;
    roundoff = (fabs(cc) * iv) * (fabs(cm) * iv) <= 1e-10;
  }
  if (between || roundoff) {
    fired = false;
    return vl;
  }
  fired = true;
  const double dm = (vm2 - vm1) - (vm1 - v0);
  const double d0 = (vm1 - v0) - (v0 - vp1);
  const double dp = (v0 - vp1) - (vp1 - vp2);
  const double cs = fmax(fabs(dm), fmax(fabs(d0), fabs(dp)));
  double d4ph = 0.0, d4mh = 0.0;
  if (cs > 0.0) {
    const double ic = 1.0 / cs;
    const double dms = dm * ic, d0s = d0 * ic, dps = dp * ic;
    d4ph = cs * minmod4(4.0 * d0s - dps, 4.0 * dps - d0s, d0s, dps);
    d4mh = cs * minmod4(4.0 * d0s - dms, 4.0 * dms - d0s, d0s, dms);
  }
  const double v_ul = v0 + 4.0 * dmn;
  const double v_av = 0.5 * v0 + 0.5 * vp1;
  const double v_md = v_av - 0.5 * d4ph;
  const double v_lc = v0 + 0.5 * dmn + (4.0 / 3.0) * d4mh;
  const double vmin = fmax(fmin(fmin(v0, vp1), v_md), fmin(fmin(v0, v_ul), v_lc));
  const double vmax = fmin(fmax(fmax(v0, vp1), v_md), fmax(fmax(v0, v_ul), v_lc));
  return vl + minmod2(vmin - vl, vmax - vl);
}
// mp_limiter.hpp:182-224: the unlimited MP interpolation of the W-point
// stencil v[0..W-1] to the face, W = 5 (MP5) or 7 (MP7).  The reference
// divides every term by the stencil's largest magnitude first, which only
// guards binary64 overflow for values near 1e305 (outside every
// configuration here); the weights are applied directly, summed as a shallow
// tree (two-term FMA pairs) rather than one dependent chain, a
// rounding-level difference.
template <int W>
__device__ __forceinline__ double mp_interp_plain(const double* v) {
  if (W == 5) {
    const double a = fma(-13.0, v[1], 2.0 * v[0]);
    const double b = fma(27.0, v[3], 47.0 * v[2]);
    return ((a + b) + (-3.0 * v[4])) * (1.0 / 60.0);
  }
  const double a = fma(25.0, v[1], -3.0 * v[0]);
  const double b = fma(319.0, v[3], -101.0 * v[2]);
  const double c = fma(-38.0, v[5], 214.0 * v[4]);
  return ((a + b) + (c + 4.0 * v[6])) * (1.0 / 420.0);
}

template <int W>
__device__ __forceinline__ double mp_recon(const double* v, bool& fired) {
  const double vl = mp_interp_plain<W>(v);
  constexpr int o = W == 5 ? 0 : 1;
  return mp_limit(vl, v[o], v[o + 1], v[o + 2], v[o + 3], v[o + 4], fired);
}

// ---- HLLD: numerics/hlld_core.hpp ----------------------------------------
// hlld_core.hpp:123-153, from the state, its pressure and 1/rho
__device__ __forceinline__ Fx physical_flux_xp(const St& u, double p, double ir) {
  const double vx = u.mx * ir, vy = u.my * ir, vz = u.mz * ir;
  const double hbn = 0.5 * (u.bx * u.bx);
  const double hbt = 0.5 * (u.by * u.by + u.bz * u.bz);
  Fx f;
  f.rho = u.mx;
  f.mx = u.mx * vx + p + u.by * (0.5 * u.by) + u.bz * (0.5 * u.bz) + u.bx * (-0.5 * u.bx);
  f.my = u.mx * vy + u.bx * (-u.by);
  f.mz = u.mx * vz + u.bx * (-u.bz);
  const double h = ((u.E - hbn) + p) + hbt;
  const double tvb = vy * u.by + vz * u.bz;
  f.E = vx * h + u.bx * (-tvb);
  f.bx = 0.0;
  f.by = u.by * vx + u.bx * (-vy);
  f.bz = u.bz * vx + u.bx * (-vz);
  return f;
}
__device__ __forceinline__ Fx physical_flux_x(const St& u, double gamma) {
  const double ir = 1.0 / u.rho;
  return physical_flux_xp(u, pressure_f(u, gamma, ir), ir);
}
__device__ __forceinline__ bool flux_finite(const Fx& f) {
  return isfinite(f.rho) && isfinite(f.mx) && isfinite(f.my) && isfinite(f.mz) &&
         isfinite(f.E) && isfinite(f.by) && isfinite(f.bz);
}
// hlld_core.hpp:157-192
__device__ __noinline__ Fx hll_flux_x(const St& L, const St& R, double sl, double sr,
                                      double gamma) {
  const Fx fl = physical_flux_x(L, gamma);
  const Fx fr = physical_flux_x(R, gamma);
  if (sl >= 0.0) return fl;
  if (sr <= 0.0) return fr;
  const double ss = fmax(fabs(sl), fabs(sr));
  if (!(ss > 0.0) || !isfinite(ss)) return fl;
  const double sln = sl / ss, srn = sr / ss;
  const double den = srn - sln;
  if (!(den > 0.0) || !isfinite(den)) return fl;
  const double wl = srn / den, wr = -sln / den;
  const double dis = ss * (sln * srn / den);
  Fx f;
  f.rho = wl * fl.rho + wr * fr.rho + dis * (R.rho - L.rho);
  f.mx = wl * fl.mx + wr * fr.mx + dis * (R.mx - L.mx);
  f.my = wl * fl.my + wr * fr.my + dis * (R.my - L.my);
  f.mz = wl * fl.mz + wr * fr.mz + dis * (R.mz - L.mz);
  f.E = wl * fl.E + wr * fr.E + dis * (R.E - L.E);
  f.bx = 0.0;
  f.by = wl * fl.by + wr * fr.by + dis * (R.by - L.by);
  f.bz = wl * fl.bz + wr * fr.bz + dis * (R.bz - L.bz);
  return f;
}
// hlld_core.hpp:200-210
__device__ __forceinline__ Fx lf_flux_x(const St& L, const St& R, double gamma) {
  const double irl = 1.0 / L.rho, irr = 1.0 / R.rho;
  const double aL = fabs(L.mx * irl) + fast_x_f(L, pressure_f(L, gamma, irl), irl, gamma);
  const double aR = fabs(R.mx * irr) + fast_x_f(R, pressure_f(R, gamma, irr), irr, gamma);
  const double a = (aL > aR) ? aL : aR;
  return hll_flux_x(L, R, -a, a, gamma);
}
__device__ __forceinline__ bool same_state(const St& a, const St& b) {
  return a.rho == b.rho && a.mx == b.mx && a.my == b.my && a.mz == b.mz && a.E == b.E &&
         a.bx == b.bx && a.by == b.by && a.bz == b.bz;
}

// hlld_core.hpp:213-457 (B0 inactive), with the reciprocal densities of the
// two states supplied (irl = 1 / Lin.rho, irr = 1 / Rin.rho).
__device__ __forceinline__ Fx hlld_flux_x(const St& Lin, const St& Rin, double gamma,
                                          double irl, double irr) {
  const double rel = 64.0 * kEps;
  if (same_state(Lin, Rin)) return physical_flux_xp(Lin, pressure_f(Lin, gamma, irl), irl);
  const double bn = 0.5 * Lin.bx + 0.5 * Rin.bx;
  St L = Lin, R = Rin;
  const double hbn2 = 0.5 * (bn * bn);
  L.E = (L.E - 0.5 * (L.bx * L.bx)) + hbn2;
  R.E = (R.E - 0.5 * (R.bx * R.bx)) + hbn2;
  L.bx = bn;
  R.bx = bn;
  const bool bn2_ok = hbn2 <= 0.5 * 1.7976931348623157e308;
  const double bn2 = bn2_ok ? 2.0 * hbn2 : 0.0;
  const double vxL = L.mx * irl, vyL = L.my * irl, vzL = L.mz * irl;
  const double vxR = R.mx * irr, vyR = R.my * irr, vzR = R.mz * irr;
  const double pL = pressure_f(L, gamma, irl), pR = pressure_f(R, gamma, irr);
  const double ptL = pL + 0.5 * (L.bx * L.bx + L.by * L.by + L.bz * L.bz);
  const double ptR = pR + 0.5 * (R.bx * R.bx + R.by * R.by + R.bz * R.bz);
  const double cfL = fast_x_f(L, pL, irl, gamma), cfR = fast_x_f(R, pR, irr, gamma);
  const double cfm = (cfL > cfR) ? cfL : cfR;
  const double sl = ((vxL < vxR) ? vxL : vxR) - cfm;
  const double sr = ((vxL > vxR) ? vxL : vxR) + cfm;
  if (sl >= 0.0) return physical_flux_xp(L, pL, irl);
  if (sr <= 0.0) return physical_flux_xp(R, pR, irr);
  if (!bn2_ok || !isfinite(ptL) || !isfinite(ptR)) return hll_flux_x(L, R, sl, sr, gamma);
  auto resolved = [&](double v, double s) { return isfinite(v) && fabs(v) > rel * (s + kTiny); };
  const double aR = (sr - vxR) * R.rho, aL = (sl - vxL) * L.rho;
  const double dM = aR - aL;
  if (!resolved(dM, fabs(aR) + fabs(aL))) return hll_flux_x(L, R, sl, sr, gamma);
  const double sm = (aR * vxR - aL * vxL - ptR + ptL) / dM;
  if (!isfinite(sm)) return hll_flux_x(L, R, sl, sr, gamma);
  const double pts = (aR * ptL - aL * ptR + L.rho * R.rho * (sr - vxR) * (sl - vxL) * (vxR - vxL)) / dM;
  if (!isfinite(pts)) return hll_flux_x(L, R, sl, sr, gamma);
  const double dLs = sl - sm, dRs = sr - sm;
  const double ws = fabs(sl) + fabs(sr) + fabs(sm);
  if (!resolved(dLs, ws) || !resolved(dRs, ws)) return hll_flux_x(L, R, sl, sr, gamma);
  const double rhoLs = L.rho * (sl - vxL) / dLs;
  const double rhoRs = R.rho * (sr - vxR) / dRs;
  if (!(rhoLs > 0.0) || !(rhoRs > 0.0)) return hll_flux_x(L, R, sl, sr, gamma);

  // Single-star states (hlld_core.hpp:306-346)
  double vysL, vzsL, bysL, bzsL, EsL, vysR, vzsR, bysR, bzsR, EsR;
  {
    const double smv = sl - vxL;
    const double t = L.rho * smv * (sl - sm);
    const double den = t - bn2;
    if (!resolved(den, fabs(t) + bn2)) return hll_flux_x(L, R, sl, sr, gamma);
    const double id = 1.0 / den;
    const double fac = bn * (sm - vxL) * id;
    vysL = vyL - L.by * fac;
    vzsL = vzL - L.bz * fac;
    const double bc = (L.rho * smv * smv - bn2) * id;
    bysL = L.by * bc;
    bzsL = L.bz * bc;
    const double vb = vxL * L.bx + vyL * L.by + vzL * L.bz;
    const double vbs = sm * bn + vysL * bysL + vzsL * bzsL;
    EsL = (smv * L.E - ptL * vxL + pts * sm + bn * (vb - vbs)) / (sl - sm);
  }
  {
    const double smv = sr - vxR;
    const double t = R.rho * smv * (sr - sm);
    const double den = t - bn2;
    if (!resolved(den, fabs(t) + bn2)) return hll_flux_x(L, R, sl, sr, gamma);
    const double id = 1.0 / den;
    const double fac = bn * (sm - vxR) * id;
    vysR = vyR - R.by * fac;
    vzsR = vzR - R.bz * fac;
    const double bc = (R.rho * smv * smv - bn2) * id;
    bysR = R.by * bc;
    bzsR = R.bz * bc;
    const double vb = vxR * R.bx + vyR * R.by + vzR * R.bz;
    const double vbs = sm * bn + vysR * bysR + vzsR * bzsR;
    EsR = (smv * R.E - ptR * vxR + pts * sm + bn * (vb - vbs)) / (sr - sm);
  }
  const St usL{rhoLs, rhoLs * sm, rhoLs * vysL, rhoLs * vzsL, EsL, bn, bysL, bzsL};
  const St usR{rhoRs, rhoRs * sm, rhoRs * vysR, rhoRs * vzsR, EsR, bn, bysR, bzsR};
  const double sqL = sqrt(rhoLs), sqR = sqrt(rhoRs);
  const double saL = sm - fabs(bn) / sqL;
  const double saR = sm + fabs(bn) / sqR;
  // (the reference forms both; only the upwind side's single-star state is
  // needed below, the other enters the double-star average)
  const bool negl = bn2 <= rel * (fabs(pts) + fabs(ptL) + fabs(ptR) + kTiny);
  auto star_flux = [&](const St& U, const St& us, double s, double f_rho, double f_mx,
                       double f_my, double f_mz, double f_E, double f_by, double f_bz) {
    Fx f;
    f.rho = f_rho + s * (us.rho - U.rho);
    f.mx = f_mx + s * (us.mx - U.mx);
    f.my = f_my + s * (us.my - U.my);
    f.mz = f_mz + s * (us.mz - U.mz);
    f.E = f_E + s * (us.E - U.E);
    f.bx = 0.0;
    f.by = f_by + s * (us.by - U.by);
    f.bz = f_bz + s * (us.bz - U.bz);
    return f;
  };
  const bool left_side = negl ? (sl <= 0.0 && 0.0 <= sm) : (0.0 <= sm);
  const St& U = left_side ? L : R;
  const Fx fU = left_side ? physical_flux_xp(L, pL, irl) : physical_flux_xp(R, pR, irr);
  if (negl) {
    const Fx f = left_side ? star_flux(L, usL, sl, fU.rho, fU.mx, fU.my, fU.mz, fU.E, fU.by, fU.bz)
                           : star_flux(R, usR, sr, fU.rho, fU.mx, fU.my, fU.mz, fU.E, fU.by, fU.bz);
    if (!isfinite(f.rho) || !isfinite(f.E)) return hll_flux_x(L, R, sl, sr, gamma);
    return f;
  }
  // Double-star states (hlld_core.hpp:379-411)
  const double isum = 1.0 / (sqL + sqR);
  const double sg = (bn >= 0.0) ? 1.0 : -1.0;
  const double vyss = (sqL * vysL + sqR * vysR + (bysR - bysL) * sg) * isum;
  const double vzss = (sqL * vzsL + sqR * vzsR + (bzsR - bzsL) * sg) * isum;
  const double byss = (sqL * bysR + sqR * bysL + sqL * sqR * (vysR - vysL) * sg) * isum;
  const double bzss = (sqL * bzsR + sqR * bzsL + sqL * sqR * (vzsR - vzsL) * sg) * isum;
  Fx f;
  if (left_side) {
    if (0.0 <= saL) {
      f = star_flux(L, usL, sl, fU.rho, fU.mx, fU.my, fU.mz, fU.E, fU.by, fU.bz);
    } else {
      const double vbss = sm * bn + vyss * byss + vzss * bzss;
      const double vbs = sm * bn + vysL * bysL + vzsL * bzsL;
      const double Ess = EsL - sqL * sg * (vbs - vbss);
      const St uss{rhoLs, rhoLs * sm, rhoLs * vyss, rhoLs * vzss, Ess, bn, byss, bzss};
      f.rho = fU.rho + saL * (uss.rho - usL.rho) + sl * (usL.rho - L.rho);
      f.mx = fU.mx + saL * (uss.mx - usL.mx) + sl * (usL.mx - L.mx);
      f.my = fU.my + saL * (uss.my - usL.my) + sl * (usL.my - L.my);
      f.mz = fU.mz + saL * (uss.mz - usL.mz) + sl * (usL.mz - L.mz);
      f.E = fU.E + saL * (uss.E - usL.E) + sl * (usL.E - L.E);
      f.bx = 0.0;
      f.by = fU.by + saL * (uss.by - usL.by) + sl * (usL.by - L.by);
      f.bz = fU.bz + saL * (uss.bz - usL.bz) + sl * (usL.bz - L.bz);
    }
  } else {
    if (0.0 <= saR) {
      const double vbss = sm * bn + vyss * byss + vzss * bzss;
      const double vbs = sm * bn + vysR * bysR + vzsR * bzsR;
      const double Ess = EsR + sqR * sg * (vbs - vbss);
      const St uss{rhoRs, rhoRs * sm, rhoRs * vyss, rhoRs * vzss, Ess, bn, byss, bzss};
      f.rho = fU.rho + saR * (uss.rho - usR.rho) + sr * (usR.rho - R.rho);
      f.mx = fU.mx + saR * (uss.mx - usR.mx) + sr * (usR.mx - R.mx);
      f.my = fU.my + saR * (uss.my - usR.my) + sr * (usR.my - R.my);
      f.mz = fU.mz + saR * (uss.mz - usR.mz) + sr * (usR.mz - R.mz);
      f.E = fU.E + saR * (uss.E - usR.E) + sr * (usR.E - R.E);
      f.bx = 0.0;
      f.by = fU.by + saR * (uss.by - usR.by) + sr * (usR.by - R.by);
      f.bz = fU.bz + saR * (uss.bz - usR.bz) + sr * (usR.bz - R.bz);
    } else {
      f = star_flux(R, usR, sr, fU.rho, fU.mx, fU.my, fU.mz, fU.E, fU.by, fU.bz);
    }
  }
  if (!flux_finite(f)) return hll_flux_x(L, R, sl, sr, gamma);
  return f;
}

__device__ __forceinline__ Fx hlld_flux_x(const St& Lin, const St& Rin, double gamma) {
  return hlld_flux_x(Lin, Rin, gamma, 1.0 / Lin.rho, 1.0 / Rin.rho);
}

// Face-normal Riemann flux in the lab frame (mhd_face_quadrature.hpp:173-185),
// irl / irr = 1 / rho of the two states.
template <int DIR>
__device__ __forceinline__ Fx riemann(const St& l, const St& r, bool lf, double gamma,
                                      double irl, double irr) {
  const St a = DIR == 0 ? l : swap_xy(l);
  const St b = DIR == 0 ? r : swap_xy(r);
  Fx f = lf ? lf_flux_x(a, b, gamma) : hlld_flux_x(a, b, gamma, irl, irr);
  if (DIR == 1) {
    const double t = f.mx;
    f.mx = f.my;
    f.my = t;
    const double u = f.bx;
    f.bx = f.by;
    f.by = u;
  }
  return f;
}
template <int DIR>
__device__ __forceinline__ Fx riemann(const St& l, const St& r, bool lf, double gamma) {
  return riemann<DIR>(l, r, lf, gamma, 1.0 / l.rho, 1.0 / r.rho);
}

// ---- transverse quadrature: numerics/finite_volume_quadrature.hpp:12-68 --
__constant__ double c_gauss3[3] = {5.0 / 18.0, 4.0 / 9.0, 5.0 / 18.0};
__constant__ double c_gauss4[4] = {0.173927422568726925, 0.326072577431273103,
                                   0.326072577431273103, 0.173927422568726925};
__constant__ double c_point5[3][5] = {
    {-0.0392523473402346598, 0.312987195324173573, 0.910833333333333384,
     -0.216320528657506839, 0.0317523473402346601},
    {0.00468749999999999983, -0.0604166666666666671, 1.11145833333333344,
     -0.0604166666666666671, 0.00468749999999999983},
    {0.0317523473402346601, -0.216320528657506839, 0.910833333333333384,
     0.312987195324173573, -0.0392523473402346598}};
__constant__ double c_point7[4][7] = {
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

// Weighted sum with the exact constant shortcut: all samples equal to the
// centre one return it unchanged (finite_volume_quadrature.hpp:55-68).
template <int N>
__device__ __forceinline__ double wsum(const double* w, const double* s) {
  // the centre is not compared with itself: a NaN centre equals no other
  // sample either, so the decision is the same
  const double ref = s[N / 2];
  bool constant = true;
#pragma unroll
  for (int q = 0; q < N; ++q)
    if (q != N / 2) constant = constant && (s[q] == ref);
  if (constant) return ref;
  double sum = w[0] * s[0];
#pragma unroll
  for (int q = 1; q < N; ++q) sum += w[q] * s[q];
  return sum;
}

// Compile-time selected quadrature weights (constant-bank operands).
template <int ORDER>
__device__ __forceinline__ double point_w(int q, int t) {
  return ORDER == 5 ? c_point5[q][t] : c_point7[q][t];
}
template <int ORDER>
__device__ __forceinline__ double gauss_w(int q) {
  return ORDER == 5 ? c_gauss3[q] : c_gauss4[q];
}
// Point value at Gauss node q from N = 5/7 transverse averages s[].
template <int ORDER>
__device__ __forceinline__ double point_value(int q, const double* s) {
  constexpr int N = ORDER == 5 ? 5 : 7;
  double w[N];
#pragma unroll
  for (int t = 0; t < N; ++t) w[t] = point_w<ORDER>(q, t);
  return wsum<N>(w, s);
}
// Point values at all Q = 3/4 Gauss nodes from the same N transverse
// averages: point_value at each node, with the constant shortcut (the same
// decision at every node) tested once.
template <int ORDER>
__device__ __forceinline__ void point_values(const double* s, double* out) {
  constexpr int N = ORDER == 5 ? 5 : 7, Q = ORDER == 5 ? 3 : 4;
  bool constant = true;
#pragma unroll
  for (int t = 0; t < N; ++t)
    if (t != N / 2) constant = constant && (s[t] == s[N / 2]);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    double v = s[N / 2];
    if (!constant) {
      v = point_w<ORDER>(q, 0) * s[0];
#pragma unroll
      for (int t = 1; t < N; ++t) v += point_w<ORDER>(q, t) * s[t];
    }
    out[q] = v;
  }
}
// Gauss average of Q = 3/4 point values.
template <int ORDER>
__device__ __forceinline__ double gauss_avg(const double* s) {
  constexpr int Q = ORDER == 5 ? 3 : 4;
  double w[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) w[q] = gauss_w<ORDER>(q);
  return wsum<Q>(w, s);
}

}  // namespace qb
