// sm_100a kernels of the 2-D ideal-MHD SSP-RK3 step (FP64).
//
// One RK stage is a short pipeline of grid-wide kernels whose intermediates
// round-trip through L2/HBM (the step is FP64-compute-bound, so the extra
// traffic is cheap next to the recomputation a fully fused tile would need):
//
//   colloc_check   cell-collocated B of the stage input (computed once per
//                  state instead of once per load) + admissibility of the
//                  previous candidate + preflights of the live state
//   reconstruct    MP5/MP7 characteristic L/R face states, one face/thread
//   face_flux      Gauss-point HLLD -> face flux, face E_z (the same solve),
//                  no-jump proof and, on stage 0, the CFL signal speed
//   cell_emf       cell-average E_z + (stage 0) the dt max-reduction
//   corner_emf     upwind CT corner E_z
//   update         flux difference + EMF curl + Shu-Osher combine, fused
//   fill_ghosts    boundary closure of the new state
//
// dt lives in device memory: the stage-0 update reads it, so a whole step
// (or many) runs without a host round trip and can be captured in a graph.
#include "mhd_device.cuh"
#include "mhd_kernels.cuh"
#include "tc.cuh"

#include <cudaTypedefs.h>

#include <cooperative_groups.h>
#include <cooperative_groups/reduce.h>

#include <algorithm>
#include <mutex>
#include <vector>

namespace qb {

namespace cg = cooperative_groups;

namespace {

constexpr int kBX = 32;  // block x (coalesced along i)


// Corner/face-table index map (reference mhd_ct.hip:126-139): periodic axes
// wrap into [0,n); physical sides clamp into [0,n].
__device__ __forceinline__ int face_index(int q, int n, int lo, int hi) {
  if (lo == 0 && hi == 0) {
    int w = q % n;
    if (w < 0) w += n;
    return w;
  }
  if (q < 0) return 0;
  if (q > n) return n;
  return q;
}

__device__ __forceinline__ bool in_pad(const Grid& g, int i, int j) {
  return i >= -g.ng && i < g.nx + g.ng && j >= -g.ng && j < g.ny + g.ng;
}

// Cell state with the high-order collocated field (reference
// mhd_staggering.hpp:321-338, collocation order 0).
__device__ __forceinline__ St load_cell(const StateP& u, long long k) {
  return St{__ldg(u.c[0] + k), __ldg(u.c[1] + k), __ldg(u.c[2] + k), __ldg(u.c[3] + k),
            __ldg(u.c[4] + k), __ldg(u.bxc + k), __ldg(u.byc + k), __ldg(u.c[7] + k)};
}

// Two-face average used by the low-order retry operator
// (mhd_staggering.hpp:243-254): the outermost high ghost keeps its sole face.
__device__ __forceinline__ double low_order_b(const double* f, const Grid& g, int cell,
                                              int hi, long long k, long long step) {
  const double lo_face = f[k];
  if (cell >= hi) return lo_face;
  return __dmul_rn(__dadd_rn(lo_face, f[k + step]), 0.5);  // = / 2 exactly
}
__device__ __forceinline__ St load_cell1(const StateP& u, const Grid& g, int i, int j) {
  const long long k = g.idx(i, j);
  St s{u.c[0][k], u.c[1][k], u.c[2][k], u.c[3][k], u.c[4][k], 0.0, 0.0, u.c[7][k]};
  s.bx = low_order_b(u.c[5], g, i, g.nx + g.ng - 1, k, 1);
  s.by = low_order_b(u.c[6], g, j, g.ny + g.ng - 1, k, g.pitch);
  return s;
}

// ---- face -> cell collocation (mhd_staggering.hpp:77-236) -----------------
__constant__ double c_f2c6[6] = {11, -93, 802, 802, -93, 11};
__constant__ double c_f2c8[8] = {-191, 1879, -9531, 68323, 68323, -9531, 1879, -191};
__constant__ double c_f2c4[4] = {-1, 13, 13, -1};
__constant__ double c_bary8[8] = {1, -7, 21, -35, 35, -21, 7, -1};
__constant__ double c_bary6[6] = {1, -5, 10, -10, 5, -1};
__constant__ double c_bary4[4] = {1, -3, 3, -1};
__constant__ double c_gx[4] = {0.0694318442029737124, 0.3300094782075718676,
                               0.6699905217924281324, 0.9305681557970262876};
__constant__ double c_gw[4] = {0.1739274225687269287, 0.3260725774312730713,
                               0.3260725774312730713, 0.1739274225687269287};

// Width-W collocation of the face samples f[k0 + step*q] for q = start..start+W-1
// at cell `cell` (W = 4, 6, 8 for 2, 3, 4 ghost layers).
template <int W>
__device__ double face_to_cell(const double* f, long long base, long long step, int cell,
                               int lo, int hi) {
  double cw[W];
#pragma unroll
  for (int k = 0; k < W; ++k) cw[k] = W == 8 ? c_f2c8[k] : W == 6 ? c_f2c6[k] : c_f2c4[k];
  const double den = W == 8 ? 120960.0 : W == 6 ? 1440.0 : 24.0;
  const int cs = cell - (W / 2 - 1);
  if (cs >= lo && cs + W - 1 <= hi) {
    double x[W];
#pragma unroll
    for (int k = 0; k < W; ++k) x[k] = __ldg(f + base + step * (long long)(cs + k));
    // Exact numerator rounded once, then one division (reference
    // scaled_rational_weighted_sum): a constant collocates to itself.
    return __ddiv_rn(exact_dot<W>(cw, x), den);
  }
  // One-sided outer-ghost closure: Gauss integral of the barycentric
  // interpolant through the W nearest faces (mhd_staggering.hpp:113-173).
  int start = cs < lo ? lo : cs;
  if (start + W - 1 > hi) start = hi - W + 1;
  double bw[W];
#pragma unroll
  for (int k = 0; k < W; ++k) bw[k] = W == 8 ? c_bary8[k] : W == 6 ? c_bary6[k] : c_bary4[k];
  const double rel = double(cell - start);
  double s = 0.0, c = 0.0;
  for (int q = 0; q < 4; ++q) {
    const double x = __dadd_rn(rel, c_gx[q]);
    double ds = 0.0, dc = 0.0;
    for (int k = 0; k < W; ++k) {
      double e;
      two_sum(ds, __ddiv_rn(bw[k], __dadd_rn(x, -double(k))), ds, e);
      dc = __dadd_rn(dc, e);
    }
    const double dsum = __dadd_rn(ds, dc);
    for (int k = 0; k < W; ++k) {
      const double wb = __dmul_rn(c_gw[q], bw[k]);
      const double v = f[base + step * (long long)(start + k)];
      const double t = __ddiv_rn(__ddiv_rn(__dmul_rn(wb, v), __dadd_rn(x, -double(k))), dsum);
      double e;
      two_sum(s, t, s, e);
      c = __dadd_rn(c, e);
    }
  }
  return __dadd_rn(s, c);
}

// ---- boundary closure (mhd_boundary_hip.hip:66-218) ------------------------
__device__ __forceinline__ void ghost_src(int n, int layer, bool lo, int mode, int& gi, int& si) {
  gi = lo ? -layer : n - 1 + layer;
  if (mode == 0) si = lo ? n - layer : layer - 1;
  else if (mode == 1) si = lo ? 0 : n - 1;
  else si = lo ? layer - 1 : n - layer;
}

// One ghost layer of one boundary line.  parts: bit 0 the fluid components
// (rho, momentum, energy, bz_cell; a wall flips the normal momentum), bit 1
// the staggered field (tangential face even; the normal face by its own rule).
__device__ __forceinline__ void fill_ghost(const Grid& g, const StateP& u, int axis, bool lo,
                                           int mode, int layer, int line, int parts) {
  const int n = axis == 0 ? g.nx : g.ny;
  int gi, si;
  ghost_src(n, layer, lo, mode, gi, si);
  auto at = [&](int a) { return axis == 0 ? g.idx(a, line) : g.idx(line, a); };
  const long long kd = at(gi), ks = at(si);
  const double sn = mode == 2 ? -1.0 : 1.0;
  if (parts & 1) {
    u.c[0][kd] = u.c[0][ks];
    u.c[1][kd] = (axis == 0 ? sn : 1.0) * u.c[1][ks];
    u.c[2][kd] = (axis == 1 ? sn : 1.0) * u.c[2][ks];
    u.c[3][kd] = u.c[3][ks];
    u.c[4][kd] = u.c[4][ks];
    u.c[7][kd] = u.c[7][ks];
  }
  if (!(parts & 2)) return;
  double* bn = axis == 0 ? u.c[5] : u.c[6];
  double* bt = axis == 0 ? u.c[6] : u.c[5];
  bt[kd] = bt[ks];
  if (mode == 2) {
    if (lo) {
      bn[at(0)] = 0.0;
      bn[at(-layer)] = -bn[at(layer)];
    } else if (layer == 1) {
      bn[at(n)] = 0.0;
    } else {
      bn[at(n + layer - 1)] = -bn[at(n - (layer - 1))];
    }
  } else if (mode == 1 && !lo) {
    // the physical high face n is evolved by CT; only faces beyond it copy it
    if (layer > 1) bn[at(n - 1 + layer)] = bn[at(n)];
  } else {
    bn[kd] = sn * bn[ks];
  }
}

// axis 0: the x sides (both), all padded rows; axis 1: the y sides over all
// padded columns (run after axis 0 so the corner blocks close last).
__device__ __forceinline__ void b_fill_ghosts(const Grid& g, const StateP& u, int axis, int bx) {
  const int lines = (axis == 0 ? g.ny : g.nx) + 2 * g.ng;
  const int t = bx * blockDim.x + threadIdx.x;
  if (t >= 2 * g.ng * lines) return;
  const int side = t / (g.ng * lines);
  const int rem = t - side * g.ng * lines;
  fill_ghost(g, u, axis, side == 0, g.bc[axis * 2 + side], rem / lines + 1, rem % lines - g.ng, 3);
}

__global__ void k_fill_ghosts(Grid g, StateP u, int axis) {
  b_fill_ghosts(g, u, axis, blockIdx.x);
}

// ---- admissible convex fraction (mhd_reduce.hip:120-209) ------------------
__device__ __forceinline__ double convex_q(const St& a, const St& b, double th) {
  const double omt = 1.0 - th;
  const double rho = omt * a.rho + th * b.rho;
  if (!(rho > 0.0) || !isfinite(rho)) return -kInf;
  const double mx = omt * a.mx + th * b.mx, my = omt * a.my + th * b.my;
  const double mz = omt * a.mz + th * b.mz, e = omt * a.E + th * b.E;
  const double bx = omt * a.bx + th * b.bx, by = omt * a.by + th * b.by;
  const double bz = omt * a.bz + th * b.bz;
  const double q = (e - kin_mom(mx, my, mz, rho)) - half_sq3(bx, by, bz);
  return isfinite(q) ? q : -kInf;
}
// Internal energy certainly positive: plain arithmetic with a margin far
// above its rounding error (a few ulps of E + kinetic + magnetic), so the
// sign agrees with the reference's scaled form whenever this returns true.
__device__ __forceinline__ bool surely_admissible(const St& s) {
  if (!(isfinite(s.rho) && s.rho > 0.0 && isfinite(s.mx) && isfinite(s.my) && isfinite(s.mz) &&
        isfinite(s.E) && isfinite(s.bx) && isfinite(s.by) && isfinite(s.bz)))
    return false;
  const double kin = 0.5 * ((s.mx * s.mx + s.my * s.my + s.mz * s.mz) / s.rho);
  const double mag = 0.5 * (s.bx * s.bx + s.by * s.by + s.bz * s.bz);
  const double q = (s.E - kin) - mag;
  return isfinite(q) && q > 1e-12 * (fabs(s.E) + kin + mag);
}

__device__ double admissible_fraction(const St& a, const St& b) {
  // both end points certainly admissible: the exact path returns 1 as well
  // (convex_q at theta 0 and 1 are the end points themselves)
  if (surely_admissible(a) && surely_admissible(b)) return 1.0;
  const double qa = convex_q(a, b, 0.0);
  if (!(a.rho > 0.0) || !(qa > 0.0) || !isfinite(a.rho) || !isfinite(qa)) return 0.0;
  if (!(isfinite(b.rho) && isfinite(b.mx) && isfinite(b.my) && isfinite(b.mz) &&
        isfinite(b.E) && isfinite(b.bx) && isfinite(b.by) && isfinite(b.bz)))
    return 0.0;
  double hi = 1.0;
  if (b.rho <= 0.0) {
    const double den = a.rho - b.rho;
    hi = den > 0.0 ? a.rho / den : 0.0;
    hi = fmin(fmax(hi, 0.0), 1.0);
  }
  if (convex_q(a, b, hi) > 0.0) return hi;
  double lo = 0.0;
  for (int it = 0; it < 56; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (convex_q(a, b, mid) > 0.0) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ unsigned long long dbits(double x) {
  return (unsigned long long)__double_as_longlong(x);
}

// atomicMax of non-negative double bit patterns, one atomic per group of
// converged lanes: the per-cell maxima of a developed flow hit one address
// from nearly every cell, and same-address atomics serialise in L2.  The max
// is exact and order-free, so the stored value is the per-cell one's.
__device__ __forceinline__ void atomic_max_lanes(unsigned long long* dst, unsigned long long v) {
  const cg::coalesced_group grp = cg::coalesced_threads();
  const unsigned long long m = cg::reduce(grp, v, cg::greater<unsigned long long>());
  if (grp.thread_rank() == 0 && m != 0ull) atomicMax(dst, m);
}

// ulp of a finite double as used by the solenoidality preflight
// (numerics/mhd_background_metrics.hpp:105-121).
__device__ __forceinline__ double ulp_of(double x) {
  const double m = fabs(x);
  if (!isfinite(x)) return kInf;
  if (m < kTiny) return 4.9406564584124654e-324;
  int e;
  frexp(m, &e);
  return ldexp(0.5, e - 52);
}

// Discrete div B of interior cell k relative to the directional scale
// (mhd_reduce.hip:556-700, solver mhd_solver.cpp:1196-1222): the residual
// the rounding envelope does not explain and the scale |d1| + |d2|, as bit
// patterns of non-negative doubles (0 = nothing to record; a non-finite
// stencil records an infinite residual).
__device__ __forceinline__ void divb_cell(const Grid& g, const StateP& u, long long k,
                                          int solver_owned, unsigned long long& rb,
                                          unsigned long long& sb) {
  const double bxl = u.c[5][k], bxh = u.c[5][k + 1];
  const double byl = u.c[6][k], byh = u.c[6][k + g.pitch];
  const double rdx = pow2_recip(g.dx), rdy = pow2_recip(g.dy);
  const double d1 = div_by(__dadd_rn(bxh, -bxl), g.dx, rdx);
  const double d2 = div_by(__dadd_rn(byh, -byl), g.dy, rdy);
  const double res = __dadd_rn(d1, d2);
  const double scale = __dadd_rn(fabs(d1), fabs(d2));
  const double unc = __dadd_rn(div_by(__dadd_rn(ulp_of(bxh), ulp_of(bxl)), g.dx, rdx),
                               div_by(__dadd_rn(ulp_of(byh), ulp_of(byl)), g.dy, rdy));
  bool explained;
  if (solver_owned) {
    explained = fabs(res) <= 1024.0 * unc;
  } else {
    explained = d1 != 0.0 && d2 != 0.0 && (signbit(d1) != signbit(d2)) &&
                fabs(res) <= 0.5 * scale && fabs(res) <= 1024.0 * unc;
  }
  const double r = explained ? 0.0 : fabs(res);
  const bool finite = isfinite(r) && isfinite(scale);
  rb = !finite ? dbits(kInf) : r > 0.0 ? dbits(r) : 0ull;
  sb = finite && scale > 0.0 ? dbits(scale) : 0ull;
}

// Collocate the candidate state's in-plane field (padded range) and, for
// interior cells, run the admissibility fraction against `base` and the
// live-state preflights.  theta_mask: bit0 collocation order 0, bit1 order 1,
// bit2 order 1 only when the live state's low-order anchor is admissible.
template <int W>
__device__ __forceinline__ void b_colloc_check(const Grid& g, const StateP& cand, const StateP& base, int has_base,
                                               int theta_mask, int live_checks, int solver_owned,
                                               double gamma, Ctl* ctl, int bx, int by) {
  const int i = bx * blockDim.x + threadIdx.x - g.ng;
  const int j = by * blockDim.y + threadIdx.y - g.ng;
  if (i >= g.nx + g.ng || j >= g.ny + g.ng) return;
  if (ctl->status & ~kStatusDone) return;
  const long long k = g.idx(i, j);
  const double bxc = face_to_cell<W>(cand.c[5], (long long)g.idx(0, j) - 0, 1, i, -g.ng,
                                     g.nx + g.ng - 1);
  const double byc = face_to_cell<W>(cand.c[6], (long long)g.idx(i, 0), g.pitch, j, -g.ng,
                                     g.ny + g.ng - 1);
  cand.bxc[k] = bxc;
  cand.byc[k] = byc;
  if (i < 0 || j < 0 || i >= g.nx || j >= g.ny || !g.in_window(i, j)) return;
  const St b{cand.c[0][k], cand.c[1][k], cand.c[2][k], cand.c[3][k], cand.c[4][k], bxc, byc,
             cand.c[7][k]};
  if (has_base) {
    double th = 1.0;
    if (theta_mask & 1) {
      const St a{base.c[0][k], base.c[1][k], base.c[2][k], base.c[3][k], base.c[4][k],
                 base.bxc[k], base.byc[k], base.c[7][k]};
      th = fmin(th, admissible_fraction(a, b));
    }
    const bool anchor = (theta_mask & 4) && ctl->anchor_ok != 0;
    if ((theta_mask & 2) || anchor) {
      th = fmin(th, admissible_fraction(load_cell1(base, g, i, j), load_cell1(cand, g, i, j)));
    }
    if (!(th >= 1.0)) {
      atomicMin(&ctl->theta, dbits(isfinite(th) ? th : 0.0));
      atomicOr(&ctl->status, kStatusRetry);
    }
  }
  if (live_checks) {
    const double t0 = admissible_fraction(b, b);
    if (!(t0 >= 1.0)) atomicMin(&ctl->live_theta, dbits(t0));
    const St b1 = load_cell1(cand, g, i, j);
    const double t1 = admissible_fraction(b1, b1);
    if (!(t1 >= 1.0)) atomicMin(&ctl->anchor_theta, dbits(t1));
    unsigned long long rb, sb;
    divb_cell(g, cand, k, solver_owned, rb, sb);
    atomic_max_lanes(&ctl->divb_res, rb);
    atomic_max_lanes(&ctl->divb_scale, sb);
  }
}

// Three blocks per SM: the bisection and ulp paths that are rarely taken spill
// at 80 registers, and the common path runs 22% faster than at 122 registers.
template <int W>
__global__ void __launch_bounds__(256, 3)
    k_colloc_check(Grid g, StateP cand, StateP base, int has_base, int theta_mask,
                   int live_checks, int solver_owned, double gamma, Ctl* ctl) {
  b_colloc_check<W>(g, cand, base, has_base, theta_mask, live_checks, solver_owned, gamma, ctl, blockIdx.x,
                    blockIdx.y);
}

}  // namespace

// ===========================================================================
// Reconstruction (reference mhd_reconstruct.hip:150-670)
// ===========================================================================
namespace {

template <int DIR>
__device__ __forceinline__ St rot(const St& s) {
  return DIR == 0 ? s : swap_xy(s);
}

// Replace the reconstructed normal field by the shared CT face value while
// keeping the gas pressure (mhd_reconstruct.hip:150-161).  The compensated
// sum returns E bit for bit when the two values agree.
template <int DIR>
__device__ __forceinline__ void set_normal_b(St& s, double v) {
  double& bn = DIR == 0 ? s.bx : s.by;
  s.E = crsum3(s.E, __dmul_rn(v, 0.5 * v), __dmul_rn(bn, -0.5 * bn));
  bn = v;
}

// ---- characteristic eigensystem, one wave at a time ----------------------
// Scalars of the eigensystem about a canonical (x-normal) state
// (mhd_eigensystem.hpp:63-171), shared by all seven waves.
struct Eg {
  double rho, sr, cf, cs, a, af, as, b1, b2, sbn, vn, vt1, vt2, bt1, bt2;
  double ia2, ra2, gm1, hv2, ir, isr, igm;
};
constexpr double kRs2 = 0.7071067811865475;  // 1/sqrt(2) rounded

// The magnetosonic speeds and the fast / slow normalisations keep the
// reference's scaled forms and uncontracted products: where the transverse
// field vanishes, af^2 is a difference of nearly equal squares and af its
// square root, so a one-ulp change of any input moves af by ~1e-8 and the
// face states by ~1e-11.  Quantities that feed only the eigenvector
// entries (velocities, transverse unit vector, 1/a^2, |v|^2/2) share one
// reciprocal each instead of a division per term (a rounding-level
// difference).
__device__ __forceinline__ Eg eig_scalars(const St& s, double gamma) {
  Eg e;
  const double ir = 1.0 / s.rho;
  const Pr w{s.rho, s.mx * ir, s.my * ir, s.mz * ir, pressure(s, gamma), s.bx, s.by, s.bz};
  e.rho = w.rho;
  const double p = w.p > 0.0 ? w.p : 0.0;
  e.sr = sqrt(e.rho);
  e.bt1 = w.by;
  e.bt2 = w.bz;
  double cax, ca;
  magnetosonic(e.rho, p, w.bx, w.by, w.bz, gamma, e.cf, e.cs, e.a, cax, ca);
  {
    const double sc = e.cf > 0.0 ? e.cf : 1.0;
    const double cfn = e.cf / sc, csn = e.cs / sc, an = e.a / sc;
    const double den = sub(mul(cfn, cfn), mul(csn, csn));
    if (den <= mul(64.0 * kEps, add(mul(cfn, cfn), mul(csn, csn)))) {
      e.af = kRs2;
      e.as = kRs2;
    } else {
      const double af2 = sub(mul(an, an), mul(csn, csn)) / den;
      const double as2 = sub(mul(cfn, cfn), mul(an, an)) / den;
      e.af = sqrt(af2 < 0.0 ? 0.0 : af2);
      e.as = sqrt(as2 < 0.0 ? 0.0 : as2);
    }
  }
  {
    const double bt = scaled_norm3(w.by, w.bz, 0.0);
    const double fs = e.a > ca ? e.a : ca;
    if (bt == 0.0 || bt / e.sr <= 64.0 * kEps * (fs + kTiny)) {
      e.b1 = kRs2;
      e.b2 = kRs2;
    } else {
      const double ibt = 1.0 / bt;
      e.b1 = w.by * ibt;
      e.b2 = w.bz * ibt;
    }
  }
  e.sbn = w.bx >= 0.0 ? 1.0 : -1.0;
  e.vn = w.vx;
  e.vt1 = w.vy;
  e.vt2 = w.vz;
  const double ia = e.a > 0.0 ? 1.0 / e.a : 0.0;
  e.ia2 = ia * ia;
  e.ra2 = gamma * p;
  e.gm1 = gamma - 1.0;
  e.hv2 = 0.5 * ((e.vn * e.vn + e.vt1 * e.vt1) + e.vt2 * e.vt2);
  e.ir = ir;
  e.isr = 1.0 / e.sr;
  e.igm = 1.0 / e.gm1;
  return e;
}

// Primitive left row and right column of wave k (mhd_eigensystem.hpp:176-320);
// k = 7 (the spare lane) gets zeros.
__device__ __forceinline__ void wave_vectors(const Eg& e, int k, double* lp, double* rp) {
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    lp[v] = 0.0;
    rp[v] = 0.0;
  }
  const double rho = e.rho;
  const double qf = e.cf * e.af * e.sbn, qs = e.cs * e.as * e.sbn;
  const double Af = e.a * e.af * e.sr, As = e.a * e.as * e.sr;
  const double Nf = 0.5 * e.ia2, s2 = kRs2;
  if (k == 0 || k == 6) {
    rp[0] = rho * e.af;
    rp[1] = k == 0 ? -e.af * e.cf : e.af * e.cf;
    rp[2] = k == 0 ? qs * e.b1 : -qs * e.b1;
    rp[3] = k == 0 ? qs * e.b2 : -qs * e.b2;
    rp[4] = e.af * e.ra2;
    rp[5] = As * e.b1;
    rp[6] = As * e.b2;
    lp[1] = k == 0 ? -Nf * e.af * e.cf : Nf * e.af * e.cf;
    lp[2] = k == 0 ? Nf * qs * e.b1 : -Nf * qs * e.b1;
    lp[3] = k == 0 ? Nf * qs * e.b2 : -Nf * qs * e.b2;
    lp[4] = Nf * e.af * e.ir;
    lp[5] = Nf * As * e.b1 * e.ir;
    lp[6] = Nf * As * e.b2 * e.ir;
  } else if (k == 1 || k == 5) {
    rp[2] = -e.b2 * s2;
    rp[3] = e.b1 * s2;
    rp[5] = k == 1 ? -e.sbn * e.b2 * s2 * e.sr : e.sbn * e.b2 * s2 * e.sr;
    rp[6] = k == 1 ? e.sbn * e.b1 * s2 * e.sr : -e.sbn * e.b1 * s2 * e.sr;
    lp[2] = -e.b2 * s2;
    lp[3] = e.b1 * s2;
    lp[5] = k == 1 ? -e.sbn * e.b2 * s2 * e.isr : e.sbn * e.b2 * s2 * e.isr;
    lp[6] = k == 1 ? e.sbn * e.b1 * s2 * e.isr : -e.sbn * e.b1 * s2 * e.isr;
  } else if (k == 2 || k == 4) {
    rp[0] = rho * e.as;
    rp[1] = k == 2 ? -e.as * e.cs : e.as * e.cs;
    rp[2] = k == 2 ? -qf * e.b1 : qf * e.b1;
    rp[3] = k == 2 ? -qf * e.b2 : qf * e.b2;
    rp[4] = e.as * e.ra2;
    rp[5] = -Af * e.b1;
    rp[6] = -Af * e.b2;
    lp[1] = k == 2 ? -Nf * e.as * e.cs : Nf * e.as * e.cs;
    lp[2] = k == 2 ? -Nf * qf * e.b1 : Nf * qf * e.b1;
    lp[3] = k == 2 ? -Nf * qf * e.b2 : Nf * qf * e.b2;
    lp[4] = Nf * e.as * e.ir;
    lp[5] = -Nf * Af * e.b1 * e.ir;
    lp[6] = -Nf * Af * e.b2 * e.ir;
  } else if (k == 3) {
    rp[0] = 1.0;
    lp[0] = 1.0;
    lp[4] = -e.ia2;
  }
}

// One thread per face, wave loop rolled: L row and R column of each wave are
// rebuilt from the shared eigen scalars when needed, so only the stencil
// deltas stay resident.  Same arithmetic per entry as build_eig.
__device__ __forceinline__ void conserved_row_col(const Eg& e, int k, double* Lr, double* Rc) {
  double lp[7], rp[7];
  wave_vectors(e, k, lp, rp);
  const double gv = e.gm1;
  Lr[0] = (((lp[0] * 1.0 + lp[1] * (-e.vn * e.ir)) + lp[2] * (-e.vt1 * e.ir)) +
           lp[3] * (-e.vt2 * e.ir)) + lp[4] * (gv * e.hv2);
  Lr[1] = lp[1] * e.ir + lp[4] * (-gv * e.vn);
  Lr[2] = lp[2] * e.ir + lp[4] * (-gv * e.vt1);
  Lr[3] = lp[3] * e.ir + lp[4] * (-gv * e.vt2);
  Lr[4] = lp[4] * gv;
  Lr[5] = lp[4] * (-gv * e.bt1) + lp[5];
  Lr[6] = lp[4] * (-gv * e.bt2) + lp[6];
  Rc[0] = rp[0];
  Rc[1] = e.vn * rp[0] + e.rho * rp[1];
  Rc[2] = e.vt1 * rp[0] + e.rho * rp[2];
  Rc[3] = e.vt2 * rp[0] + e.rho * rp[3];
  Rc[4] = (((((e.hv2 * rp[0] + (e.rho * e.vn) * rp[1]) + (e.rho * e.vt1) * rp[2]) +
             (e.rho * e.vt2) * rp[3]) + e.igm * rp[4]) + e.bt1 * rp[5]) + e.bt2 * rp[6];
  Rc[5] = rp[5];
  Rc[6] = rp[6];
}

// Dynamic shared memory of every kernel that runs mp_pair_loop: 98 doubles
// (7 L rows + 7 R columns) per thread of a 128-thread block.
constexpr int kReconThreads = 128;
constexpr size_t kReconSmem = 98 * kReconThreads * sizeof(double);

template <int DIR, int H>
__device__ void mp_pair_loop(const StateP& u, long long k0, long long step, double gamma, St& ul,
                             St& ur, bool* fired_l = nullptr, bool* fired_r = nullptr) {
  constexpr int S = 2 * H + 2, W = 2 * H + 1;
  const St cl = load_cell(u, k0 - step), cr = load_cell(u, k0);
  St ref;
  ref.rho = 0.5 * cl.rho + 0.5 * cr.rho;
  ref.mx = 0.5 * cl.mx + 0.5 * cr.mx;
  ref.my = 0.5 * cl.my + 0.5 * cr.my;
  ref.mz = 0.5 * cl.mz + 0.5 * cr.mz;
  ref.E = 0.5 * cl.E + 0.5 * cr.E;
  ref.bx = 0.5 * cl.bx + 0.5 * cr.bx;
  ref.by = 0.5 * cl.by + 0.5 * cr.by;
  ref.bz = 0.5 * cl.bz + 0.5 * cr.bz;
  const St c = rot<DIR>(ref);
  const Eg e = eig_scalars(c, gamma);
  // All seven L rows and R columns built once into this thread's slots of
  // dynamic shared memory (kReconSmemDoubles per thread, stride = threads per
  // block), then the L R = I check (mhd_eigensystem.hpp:416-430) with R
  // resident in two halves (4 + 3).  |d| <= 1024 eps is tested as
  // d^2 <= (1024 eps)^2, the same decision since 1024 eps is a power of two
  // (and false for NaN and infinity).
  extern __shared__ double dsm[];
  const int ST = blockDim.x * blockDim.y;
  double* LR = dsm + (threadIdx.y * blockDim.x + threadIdx.x);
#pragma unroll 1
  for (int k = 0; k < 7; ++k) {
    double Lr[7], Rc[7];
    conserved_row_col(e, k, Lr, Rc);
#pragma unroll
    for (int m = 0; m < 7; ++m) {
      LR[(k * 7 + m) * ST] = Lr[m];
      LR[(49 + k * 7 + m) * ST] = Rc[m];
    }
  }
  bool usable = true;
  constexpr double kT2 = (1024.0 * kEps) * (1024.0 * kEps);
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    constexpr int kCols = 4;
    const int j0 = half * kCols, nj = half == 0 ? kCols : 7 - kCols;
    double Rm[kCols][7];
#pragma unroll
    for (int jj = 0; jj < kCols; ++jj)
#pragma unroll
      for (int m = 0; m < 7; ++m) Rm[jj][m] = jj < nj ? LR[(49 + (j0 + jj) * 7 + m) * ST] : 0.0;
#pragma unroll 1
    for (int i = 0; i < 7; ++i) {
      double Lr[7];
#pragma unroll
      for (int m = 0; m < 7; ++m) Lr[m] = LR[(i * 7 + m) * ST];
#pragma unroll
      for (int jj = 0; jj < kCols; ++jj) {
        if (jj >= nj) continue;
        double dot = 0.0;
#pragma unroll
        for (int m = 0; m < 7; ++m) dot += Lr[m] * Rm[jj][m];
        const double d = dot - (i == j0 + jj ? 1.0 : 0.0);
        usable = usable && (d * d <= kT2);
      }
    }
  }
  // stencil deltas in the canonical frame
  double u7[S][7];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const St d = rot<DIR>(load_cell(u, k0 + (long long)(s - 1 - H) * step));
    u7[s][0] = d.rho - c.rho;
    u7[s][1] = d.mx - c.mx;
    u7[s][2] = d.my - c.my;
    u7[s][3] = d.mz - c.mz;
    u7[s][4] = d.E - c.E;
    u7[s][5] = d.by - c.by;
    u7[s][6] = d.bz - c.bz;
  }
  double dl[7], dr[7];
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    dl[v] = 0.0;
    dr[v] = 0.0;
  }
#pragma unroll 1
  for (int k = 0; k < 7; ++k) {
    double Lr[7];
    if (usable) {
#pragma unroll
      for (int m = 0; m < 7; ++m) Lr[m] = LR[(k * 7 + m) * ST];
    } else {
#pragma unroll
      for (int v = 0; v < 7; ++v) Lr[v] = v == k ? 1.0 : 0.0;
    }
    double ch[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      double acc = 0.0;
#pragma unroll
      for (int v = 0; v < 7; ++v) acc += Lr[v] * u7[s][v];
      ch[s] = acc;
    }
    double win[W];
    bool f;
#pragma unroll
    for (int s = 0; s < W; ++s) win[s] = ch[s];
    const double wl = mp_recon<W>(win, f);
    if (fired_l && f) *fired_l = true;
#pragma unroll
    for (int s = 0; s < W; ++s) win[s] = ch[W - s];
    const double wr = mp_recon<W>(win, f);
    if (fired_r && f) *fired_r = true;
    double Rc[7];
    if (usable) {
#pragma unroll
      for (int m = 0; m < 7; ++m) Rc[m] = LR[(49 + k * 7 + m) * ST];
    } else {
#pragma unroll
      for (int v = 0; v < 7; ++v) Rc[v] = v == k ? 1.0 : 0.0;
    }
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      dl[v] += Rc[v] * wl;
      dr[v] += Rc[v] * wr;
    }
  }
  const St sl{c.rho + dl[0], c.mx + dl[1], c.my + dl[2], c.mz + dl[3],
              c.E + dl[4],   c.bx,         c.by + dl[5], c.bz + dl[6]};
  const St sr{c.rho + dr[0], c.mx + dr[1], c.my + dr[2], c.mz + dr[3],
              c.E + dr[4],   c.bx,         c.by + dr[5], c.bz + dr[6]};
  ul = rot<DIR>(sl);
  ur = rot<DIR>(sr);
}

// Component-wise unlimited MP interpolation of the same conserved deltas:
// the characteristic path with L = R = I and no limiter, which equals the
// characteristic result wherever the limiter accepts every wave (R L = I).
// The components are independent, so each is loaded, interpolated and
// finished before the next (few live registers); the sums are those of the
// whole-state form.
template <int DIR, int H>
__device__ void mp_pair_lin(const StateP& u, long long k0, long long step, St& ul, St& ur) {
  constexpr int S = 2 * H + 2, W = 2 * H + 1;
  double dl[8], dr[8], cv[8];
  // canonical frame: rho, m_n, m_t1, m_t2, E, b_n, b_t1, b_t2
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const double* a = v == 0 ? u.c[0]
                      : v == 1 ? (DIR == 0 ? u.c[1] : u.c[2])
                      : v == 2 ? (DIR == 0 ? u.c[2] : u.c[1])
                      : v == 3 ? u.c[3]
                      : v == 4 ? u.c[4]
                      : v == 5 ? (DIR == 0 ? u.bxc : u.byc)
                      : v == 6 ? (DIR == 0 ? u.byc : u.bxc)
                               : u.c[7];
    const double c = 0.5 * __ldg(a + k0 - step) + 0.5 * __ldg(a + k0);
    cv[v] = c;
    if (v == 5) continue;  // the normal field is not reconstructed
    double w[S];
#pragma unroll
    for (int t = 0; t < S; ++t) w[t] = __ldg(a + k0 + (long long)(t - 1 - H) * step) - c;
    dl[v] = mp_interp_plain<W>(w);
    double wr[W];
#pragma unroll
    for (int t = 0; t < W; ++t) wr[t] = w[W - t];
    dr[v] = mp_interp_plain<W>(wr);
  }
  const St sl{cv[0] + dl[0], cv[1] + dl[1], cv[2] + dl[2], cv[3] + dl[3],
              cv[4] + dl[4], cv[5],         cv[6] + dl[6], cv[7] + dl[7]};
  const St sr{cv[0] + dr[0], cv[1] + dr[1], cv[2] + dr[2], cv[3] + dr[3],
              cv[4] + dr[4], cv[5],         cv[6] + dr[6], cv[7] + dr[7]};
  ul = rot<DIR>(sl);
  ur = rot<DIR>(sr);
}

template <int DIR, int ORDER, int MODE>
__device__ __forceinline__ void finish_face(const Grid& g, const StateP& u, const IfaceP& out,
                                            double gamma, int i, int j, long long k0,
                                            long long step, St ul, St ur);

// ---- warp-cooperative characteristic MP reconstruction --------------------
// The characteristic path of mp_pair_loop with the work of one face spread
// over four lanes, lane r holding the pair of waves r and 6 - r (lane 3 the
// entropy wave alone), so that a thread carries two waves' L rows and
// projected stencils instead of all seven, and has two independent chains.
// A warp owns 32 faces:
//   phase 1  lane = face: reference state and eigen scalars -> shared memory
//   phase 2  4 rounds of 8 faces, lane = (face, wave pair): L rows and R
//            columns, the L R = I check (R columns exchanged through shared
//            memory), the stencil deltas (lane = two stencil cells),
//            projection, MP limiter on both sides, back-projection (lane =
//            components r and r + 4)
//   phase 3  lane = face: states, fallback chain, stores (finish_face)
// Every value is formed by the same operations in the same order as
// mp_pair_loop, so the two paths agree to the FMA contraction the compiler
// picks for each expression.  Four lanes per face (not seven) because the
// exchanged operands are read once per lane: each shared-memory load costs
// one wavefront per half-warp whether or not the lanes share its address.
//
// Per-warp shared memory (doubles): a face record [kRec][32] and eight group
// buffers R[7][8] followed by delta[8][7], whose first 14 slots later hold
// the projected face values w[2][7].  The R columns are padded to eight
// doubles so that the L R = I check reads them as 16-byte pairs (half the
// load instructions of scalar reads: reconstruction went 39.9 -> 37.8 ms per
// rotor 4096^2 MP7 step); the group stride of 114 doubles
// puts the eight groups' 16-byte reads on distinct banks.  Padding the
// stencil deltas the same way measured no faster.
constexpr int kRecC = 0;    // canonical reference state, 8 components
constexpr int kRecE = 8;    // 17 eigen scalars, later dl[7] and dr[7]
constexpr int kRec = 25;
constexpr int kGrpR = 0, kRS = 8, kGrpD = 56, kGrpW = 56, kGrpDoubles = 114;
constexpr int kGroups = 8;
constexpr int kWarpReconDoubles = kRec * 32 + kGroups * kGrpDoubles;
constexpr int kReconWarps = 4;
constexpr size_t kReconWarpSmem = size_t(kReconWarps) * kWarpReconDoubles * sizeof(double);

// L row and R column of wave k (k = 7: zeros) without branching on k: the
// three families are formed side by side and selected, entry for entry the
// products of wave_vectors and the sums of conserved_row_col.
__device__ __forceinline__ void wave_lr(const Eg& e, int k, double* Lr, double* Rc) {
  const double rho = e.rho;
  const double s2 = kRs2, Nf = 0.5 * e.ia2;
  // magnetosonic (k = 0, 2, 4, 6): fast for 0 and 6, slow for 2 and 4;
  // the "minus" member of each pair is k < 3
  const bool fs = (k == 0 || k == 6);
  const bool neg = k < 3;
  const double qf = e.cf * e.af * e.sbn, qs = e.cs * e.as * e.sbn;
  const double Af = e.a * e.af * e.sr, As = e.a * e.as * e.sr;
  const double al = fs ? e.af : e.as;
  const double cc = fs ? e.cf : e.cs;
  const double qq = fs ? qs : -qf;
  const double AA = fs ? As : -Af;
  const double ac = al * cc, qb1 = qq * e.b1, qb2 = qq * e.b2;
  const double nac = Nf * al * cc, nq1 = Nf * qq * e.b1, nq2 = Nf * qq * e.b2;
  // Alfven (k = 1, 5): the "minus" member is k = 1
  const double t5 = e.sbn * e.b2 * s2 * e.sr, t6 = e.sbn * e.b1 * s2 * e.sr;
  const double u5 = e.sbn * e.b2 * s2 * e.isr, u6 = e.sbn * e.b1 * s2 * e.isr;
  const double ab2 = -e.b2 * s2, ab1 = e.b1 * s2;
  const bool ms = (k & 1) == 0 && k != 7, alf = k == 1 || k == 5, ent = k == 3;
  const bool k1 = k == 1;
  double rp[7], lp[7];
  rp[0] = ms ? rho * al : (ent ? 1.0 : 0.0);
  rp[1] = ms ? (neg ? -ac : ac) : 0.0;
  rp[2] = ms ? (neg ? qb1 : -qb1) : (alf ? ab2 : 0.0);
  rp[3] = ms ? (neg ? qb2 : -qb2) : (alf ? ab1 : 0.0);
  rp[4] = ms ? al * e.ra2 : 0.0;
  rp[5] = ms ? AA * e.b1 : (alf ? (k1 ? -t5 : t5) : 0.0);
  rp[6] = ms ? AA * e.b2 : (alf ? (k1 ? t6 : -t6) : 0.0);
  lp[0] = ent ? 1.0 : 0.0;
  lp[1] = ms ? (neg ? -nac : nac) : 0.0;
  lp[2] = ms ? (neg ? nq1 : -nq1) : (alf ? ab2 : 0.0);
  lp[3] = ms ? (neg ? nq2 : -nq2) : (alf ? ab1 : 0.0);
  lp[4] = ms ? Nf * al * e.ir : (ent ? -e.ia2 : 0.0);
  lp[5] = ms ? Nf * AA * e.b1 * e.ir : (alf ? (k1 ? -u5 : u5) : 0.0);
  lp[6] = ms ? Nf * AA * e.b2 * e.ir : (alf ? (k1 ? u6 : -u6) : 0.0);
  const double gv = e.gm1;
  Lr[0] = (((lp[0] * 1.0 + lp[1] * (-e.vn * e.ir)) + lp[2] * (-e.vt1 * e.ir)) +
           lp[3] * (-e.vt2 * e.ir)) + lp[4] * (gv * e.hv2);
  Lr[1] = lp[1] * e.ir + lp[4] * (-gv * e.vn);
  Lr[2] = lp[2] * e.ir + lp[4] * (-gv * e.vt1);
  Lr[3] = lp[3] * e.ir + lp[4] * (-gv * e.vt2);
  Lr[4] = lp[4] * gv;
  Lr[5] = lp[4] * (-gv * e.bt1) + lp[5];
  Lr[6] = lp[4] * (-gv * e.bt2) + lp[6];
  Rc[0] = rp[0];
  Rc[1] = e.vn * rp[0] + e.rho * rp[1];
  Rc[2] = e.vt1 * rp[0] + e.rho * rp[2];
  Rc[3] = e.vt2 * rp[0] + e.rho * rp[3];
  Rc[4] = (((((e.hv2 * rp[0] + (e.rho * e.vn) * rp[1]) + (e.rho * e.vt1) * rp[2]) +
             (e.rho * e.vt2) * rp[3]) + e.igm * rp[4]) + e.bt1 * rp[5]) + e.bt2 * rp[6];
  Rc[5] = rp[5];
  Rc[6] = rp[6];
}

// One warp's 32 faces (lane = face; `valid` false for lanes without one).
// All lanes of the warp must call it; `ws` is the warp's shared memory.
template <int DIR, int ORDER>
__device__ void mp_faces_warp(const Grid& g, const StateP& u, const IfaceP& out, double gamma,
                              int i, int j, bool valid, double* ws) {
  constexpr int H = ORDER == 5 ? 2 : 3;
  constexpr int S = 2 * H + 2, W = 2 * H + 1;
  const unsigned lane = threadIdx.x & 31u;
  const long long step = DIR == 0 ? 1 : g.pitch;
  const long long k0 = valid ? g.idx(i, j) : 0;
  double* rec = ws;
  // phase 1: reference state and eigen scalars of this lane's face
  if (valid) {
    const St cl = load_cell(u, k0 - step), cr = load_cell(u, k0);
    St ref;
    ref.rho = 0.5 * cl.rho + 0.5 * cr.rho;
    ref.mx = 0.5 * cl.mx + 0.5 * cr.mx;
    ref.my = 0.5 * cl.my + 0.5 * cr.my;
    ref.mz = 0.5 * cl.mz + 0.5 * cr.mz;
    ref.E = 0.5 * cl.E + 0.5 * cr.E;
    ref.bx = 0.5 * cl.bx + 0.5 * cr.bx;
    ref.by = 0.5 * cl.by + 0.5 * cr.by;
    ref.bz = 0.5 * cl.bz + 0.5 * cr.bz;
    const St c = rot<DIR>(ref);
    const Eg e = eig_scalars(c, gamma);
    double* r = rec + lane;
    r[(kRecC + 0) * 32] = c.rho;
    r[(kRecC + 1) * 32] = c.mx;
    r[(kRecC + 2) * 32] = c.my;
    r[(kRecC + 3) * 32] = c.mz;
    r[(kRecC + 4) * 32] = c.E;
    r[(kRecC + 5) * 32] = c.bx;
    r[(kRecC + 6) * 32] = c.by;
    r[(kRecC + 7) * 32] = c.bz;
    const double ev[17] = {e.sr, e.cf, e.cs, e.a, e.af, e.as, e.b1, e.b2, e.sbn,
                           e.vn, e.vt1, e.vt2, e.ia2, e.ra2, e.hv2, e.ir, e.isr};
#pragma unroll
    for (int q = 0; q < 17; ++q) r[(kRecE + q) * 32] = ev[q];
  }
  const unsigned vmask = __ballot_sync(0xffffffffu, valid);
  // phase 2: eight faces per round, four lanes per face
  const int gi = int(lane >> 2), rl = int(lane & 3u);
  const bool two = rl < 3;           // lanes 0-2: waves rl and 6 - rl; lane 3: wave 3
  const int ka = rl, kb = 6 - rl;    // kb == ka on lane 3
  double* grp = ws + kRec * 32 + gi * kGrpDoubles;
  const double gm1 = gamma - 1.0, igm = 1.0 / gm1;
  constexpr double kT2 = (1024.0 * kEps) * (1024.0 * kEps);
#pragma unroll 1
  for (int rd = 0; rd < 4; ++rd) {
    if (((vmask >> (8 * rd)) & 0xFFu) == 0u) continue;  // warp-uniform
    const int f = 8 * rd + gi;
    const bool on = (vmask >> f) & 1u;
    const long long kf = __shfl_sync(0xffffffffu, k0, f);
    double La[7], Lb[7];
    bool ok = true;
    if (on) {
      const double* r = rec + f;
      Eg e;
      e.rho = r[(kRecC + 0) * 32];
      e.bt1 = r[(kRecC + 6) * 32];
      e.bt2 = r[(kRecC + 7) * 32];
      e.sr = r[(kRecE + 0) * 32];
      e.cf = r[(kRecE + 1) * 32];
      e.cs = r[(kRecE + 2) * 32];
      e.a = r[(kRecE + 3) * 32];
      e.af = r[(kRecE + 4) * 32];
      e.as = r[(kRecE + 5) * 32];
      e.b1 = r[(kRecE + 6) * 32];
      e.b2 = r[(kRecE + 7) * 32];
      e.sbn = r[(kRecE + 8) * 32];
      e.vn = r[(kRecE + 9) * 32];
      e.vt1 = r[(kRecE + 10) * 32];
      e.vt2 = r[(kRecE + 11) * 32];
      e.ia2 = r[(kRecE + 12) * 32];
      e.ra2 = r[(kRecE + 13) * 32];
      e.hv2 = r[(kRecE + 14) * 32];
      e.ir = r[(kRecE + 15) * 32];
      e.isr = r[(kRecE + 16) * 32];
      e.gm1 = gm1;
      e.igm = igm;
      double Ra[7], Rb[7];
      wave_lr(e, ka, La, Ra);
      wave_lr(e, kb, Lb, Rb);
#pragma unroll
      for (int m = 0; m < 7; ++m) grp[kGrpR + ka * kRS + m] = Ra[m];
      if (two) {
#pragma unroll
        for (int m = 0; m < 7; ++m) grp[kGrpR + kb * kRS + m] = Rb[m];
      }
    }
    __syncwarp();
    // L R = I within 1024 ulp (mhd_eigensystem.hpp:416-430): this lane's L
    // rows against every R column; |d| <= 1024 eps tested as
    // d^2 <= (1024 eps)^2
    if (on) {
#pragma unroll
      for (int jc = 0; jc < 7; ++jc) {
        const double2* R2 = reinterpret_cast<const double2*>(grp + kGrpR + jc * kRS);
        const double2 p0 = R2[0], p1 = R2[1], p2 = R2[2], p3 = R2[3];
        const double R7[7] = {p0.x, p0.y, p1.x, p1.y, p2.x, p2.y, p3.x};
        double da = 0.0, db = 0.0;
#pragma unroll
        for (int m = 0; m < 7; ++m) {
          da += La[m] * R7[m];
          db += Lb[m] * R7[m];
        }
        const double ea = da - (ka == jc ? 1.0 : 0.0), eb = db - (kb == jc ? 1.0 : 0.0);
        ok = ok && (ea * ea <= kT2) && (eb * eb <= kT2);
      }
    }
    const unsigned okm = __ballot_sync(0xffffffffu, ok);
    const bool usable = ((okm >> (gi * 4)) & 0xFu) == 0xFu;
    if (on && !usable) {
#pragma unroll
      for (int v = 0; v < 7; ++v) {
        La[v] = v == ka ? 1.0 : 0.0;
        Lb[v] = v == kb ? 1.0 : 0.0;
        grp[kGrpR + ka * kRS + v] = v == ka ? 1.0 : 0.0;
        if (two) grp[kGrpR + kb * kRS + v] = v == kb ? 1.0 : 0.0;
      }
    }
    // stencil deltas in the canonical frame: lane rl loads cells rl, rl + 4
    if (on) {
      const double* r = rec + f;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int sc = rl + 4 * h;
        if (sc < S) {
          const St d = rot<DIR>(load_cell(u, kf + (long long)(sc - 1 - H) * step));
          double* dd = grp + kGrpD + sc * 7;
          dd[0] = d.rho - r[(kRecC + 0) * 32];
          dd[1] = d.mx - r[(kRecC + 1) * 32];
          dd[2] = d.my - r[(kRecC + 2) * 32];
          dd[3] = d.mz - r[(kRecC + 3) * 32];
          dd[4] = d.E - r[(kRecC + 4) * 32];
          dd[5] = d.by - r[(kRecC + 6) * 32];
          dd[6] = d.bz - r[(kRecC + 7) * 32];
        }
      }
    }
    __syncwarp();
    // projection onto this lane's waves
    double cha[S], chb[S];
    if (on) {
#pragma unroll
      for (int sc = 0; sc < S; ++sc) {
        double d7[7];
#pragma unroll
        for (int v = 0; v < 7; ++v) d7[v] = grp[kGrpD + sc * 7 + v];
        double aa = 0.0, ab = 0.0;
#pragma unroll
        for (int v = 0; v < 7; ++v) {
          aa += La[v] * d7[v];
          ab += Lb[v] * d7[v];
        }
        cha[sc] = aa;
        chb[sc] = ab;
      }
    }
    __syncwarp();  // the deltas are read; w overwrites them
    // MP limiter on both sides of both waves
    if (on) {
      double win[W];
      bool fl;
#pragma unroll
      for (int sc = 0; sc < W; ++sc) win[sc] = cha[sc];
      grp[kGrpW + ka] = mp_recon<W>(win, fl);
#pragma unroll
      for (int sc = 0; sc < W; ++sc) win[sc] = cha[W - sc];
      grp[kGrpW + 7 + ka] = mp_recon<W>(win, fl);
      if (two) {
#pragma unroll
        for (int sc = 0; sc < W; ++sc) win[sc] = chb[sc];
        grp[kGrpW + kb] = mp_recon<W>(win, fl);
#pragma unroll
        for (int sc = 0; sc < W; ++sc) win[sc] = chb[W - sc];
        grp[kGrpW + 7 + kb] = mp_recon<W>(win, fl);
      }
    }
    __syncwarp();
    // back-projection: lane rl forms components rl and rl + 4 of both sides
    if (on) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int v = rl + 4 * h;
        if (v < 7) {
          double dl = 0.0, dr = 0.0;
#pragma unroll
          for (int q = 0; q < 7; ++q) {
            const double rq = grp[kGrpR + q * kRS + v];
            dl += rq * grp[kGrpW + q];
            dr += rq * grp[kGrpW + 7 + q];
          }
          rec[(kRecE + v) * 32 + f] = dl;
          rec[(kRecE + 7 + v) * 32 + f] = dr;
        }
      }
    }
    __syncwarp();
  }
  // phase 3: this lane's face
  if (!valid) return;
  const double* r = rec + lane;
  St c;
  c.rho = r[(kRecC + 0) * 32];
  c.mx = r[(kRecC + 1) * 32];
  c.my = r[(kRecC + 2) * 32];
  c.mz = r[(kRecC + 3) * 32];
  c.E = r[(kRecC + 4) * 32];
  c.bx = r[(kRecC + 5) * 32];
  c.by = r[(kRecC + 6) * 32];
  c.bz = r[(kRecC + 7) * 32];
  double dl[7], dr[7];
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    dl[v] = r[(kRecE + v) * 32];
    dr[v] = r[(kRecE + 7 + v) * 32];
  }
  const St sl{c.rho + dl[0], c.mx + dl[1], c.my + dl[2], c.mz + dl[3],
              c.E + dl[4],   c.bx,         c.by + dl[5], c.bz + dl[6]};
  const St sr{c.rho + dr[0], c.mx + dr[1], c.my + dr[2], c.mz + dr[3],
              c.E + dr[4],   c.bx,         c.by + dr[5], c.bz + dr[6]};
  finish_face<DIR, ORDER, 0>(g, u, out, gamma, i, j, k0, step, rot<DIR>(sl), rot<DIR>(sr));
}

// ---- MUSCL-minmod in primitive variables (mhd_reconstruct.hip:93-404) ----
__device__ __forceinline__ int slope_drop(int c, int n, int lo, int hi) {
  if (lo != 0 && lo != 4 && c <= 0) return -1;
  if (hi != 0 && hi != 4 && c >= n - 1) return 1;
  return 0;
}
__device__ __forceinline__ double lim(double back, double fwd, int drop) {
  if (drop < 0) return fwd;
  if (drop > 0) return back;
  return minmod2(back, fwd);
}
__device__ __forceinline__ Pr muscl_face(const Pr& m, const Pr& c, const Pr& p, double sign,
                                         int drop) {
  const double h = 0.5 * sign;
  Pr f;
  f.rho = c.rho + h * lim(c.rho - m.rho, p.rho - c.rho, drop);
  f.vx = c.vx + h * lim(c.vx - m.vx, p.vx - c.vx, drop);
  f.vy = c.vy + h * lim(c.vy - m.vy, p.vy - c.vy, drop);
  f.vz = c.vz + h * lim(c.vz - m.vz, p.vz - c.vz, drop);
  f.p = c.p + h * lim(c.p - m.p, p.p - c.p, drop);
  f.bx = c.bx + h * lim(c.bx - m.bx, p.bx - c.bx, drop);
  f.by = c.by + h * lim(c.by - m.by, p.by - c.by, drop);
  f.bz = c.bz + h * lim(c.bz - m.bz, p.bz - c.bz, drop);
  return f;
}
template <int DIR>
__device__ void muscl_pair(const Grid& g, const StateP& u, int i, int j, long long k0,
                           long long step, double gamma, St& ul, St& ur) {
  const Pr a = to_prim(load_cell(u, k0 - 2 * step), gamma);
  const Pr b = to_prim(load_cell(u, k0 - step), gamma);
  const Pr c = to_prim(load_cell(u, k0), gamma);
  const Pr d = to_prim(load_cell(u, k0 + step), gamma);
  const int n = DIR == 0 ? g.nx : g.ny;
  const int lo = g.bc[DIR * 2], hi = g.bc[DIR * 2 + 1];
  const int pos = DIR == 0 ? i : j;
  ul = to_cons(muscl_face(a, b, c, 1.0, slope_drop(pos - 1, n, lo, hi)), gamma);
  ur = to_cons(muscl_face(b, c, d, -1.0, slope_drop(pos, n, lo, hi)), gamma);
}

// How far the limited characteristic face state departs from the unlimited
// component-wise one: the largest difference relative to the state's scale
// per group (rho; momentum against sqrt(2 rho E); E; field against
// sqrt(2 E)); +inf when not finite.
__device__ __forceinline__ float limiter_departure(const St& a, const St& b) {
  const double rs = fabs(b.rho), es = fabs(b.E);
  const double ms = sqrt(2.0 * rs * es), bs = sqrt(2.0 * es);
  double d = fabs(a.rho - b.rho) / rs;
  d = fmax(d, fabs(a.mx - b.mx) / ms);
  d = fmax(d, fabs(a.my - b.my) / ms);
  d = fmax(d, fabs(a.mz - b.mz) / ms);
  d = fmax(d, fabs(a.E - b.E) / es);
  d = fmax(d, fabs(a.bx - b.bx) / bs);
  d = fmax(d, fabs(a.by - b.by) / bs);
  d = fmax(d, fabs(a.bz - b.bz) / bs);
  return isfinite(d) ? float(d) : INFINITY;
}

// Learned-mode face list of one direction: the per-cell flags it was built
// from (a face is listed when either of its cells is flagged), the list and
// its device-resident count.
struct FaceList {
  const unsigned char* flag;
  int* list;
  int* count;
};

// One face's interface states.  MODE 0: the characteristic MP path; 1: the
// same, also recording per cell the largest departure of a limited state
// from the unlimited component-wise one (label[cell] = max, as float bits;
// the left state's stencil is centred on the left cell);
// 2: the unlimited component-wise path; a face whose unlimited states are
// not admissible is appended to `defer` for the characteristic pass that
// follows (the plain step's path for it, fallbacks included) unless it is
// listed already; 3: the characteristic path, recording per cell whether the
// MP limiter fired on any characteristic field of a state whose stencil is
// centred on it (label[cell] = 1).  Orders 1 and 2 ignore MODE.
template <int DIR, int ORDER, int MODE>
__device__ __forceinline__ void recon_face(const Grid& g, const StateP& u, const IfaceP& out,
                                           double gamma, int i, int j, int* label,
                                           FaceList defer = FaceList{}) {
  const long long k0 = g.idx(i, j);
  const long long step = DIR == 0 ? 1 : g.pitch;
  St ul, ur;
  if (ORDER <= 1) {
    ul = DIR == 0 ? load_cell1(u, g, i - 1, j) : load_cell1(u, g, i, j - 1);
    ur = load_cell1(u, g, i, j);
  } else if (ORDER == 2) {
    muscl_pair<DIR>(g, u, i, j, k0, step, gamma, ul, ur);
  } else {
    constexpr int H = ORDER == 5 ? 2 : 3;
    if constexpr (MODE == 2) {
      mp_pair_lin<DIR, H>(u, k0, step, ul, ur);
      if (!recon_admissible(ul, gamma) || !recon_admissible(ur, gamma)) {
        if (!defer.flag[k0 - step] && !defer.flag[k0])
          defer.list[atomicAdd(defer.count, 1)] = int(k0);
        return;
      }
    } else {
      bool fl = false, fr = false;
      mp_pair_loop<DIR, H>(u, k0, step, gamma, ul, ur, &fl, &fr);
      if (MODE == 3) {
        // the literal label: the MP limiter fired on some characteristic
        // field of the state whose stencil is centred on the cell
        if (fl) atomicMax(label + (k0 - step), 1);
        if (fr) atomicMax(label + k0, 1);
      }
      if (MODE == 1) {
        St ll, lr;
        mp_pair_lin<DIR, H>(u, k0, step, ll, lr);
        // non-negative floats order like their bit patterns
        atomicMax(label + (k0 - step), __float_as_int(limiter_departure(ul, ll)));
        atomicMax(label + k0, __float_as_int(limiter_departure(ur, lr)));
      }
    }
  }
  finish_face<DIR, ORDER, MODE>(g, u, out, gamma, i, j, k0, step, ul, ur);
}

// The fallback chain after the high-order states of one face
// (mhd_reconstruct.hip:514-670): MUSCL when a characteristic MP state is not
// admissible, the shared CT normal field, first order, then NaN; the states
// are written to the face's interface slots.
template <int DIR, int ORDER, int MODE>
__device__ __forceinline__ void finish_face(const Grid& g, const StateP& u, const IfaceP& out,
                                            double gamma, int i, int j, long long k0,
                                            long long step, St ul, St ur) {
  if constexpr (ORDER >= 5 && MODE != 2) {
    if (!recon_admissible(ul, gamma) || !recon_admissible(ur, gamma))
      muscl_pair<DIR>(g, u, i, j, k0, step, gamma, ul, ur);
  }
  const double bn = (DIR == 0 ? u.c[5] : u.c[6])[k0];
  set_normal_b<DIR>(ul, bn);
  set_normal_b<DIR>(ur, bn);
  if (!recon_admissible(ul, gamma) || !recon_admissible(ur, gamma)) {
    if (ORDER <= 1) {
      ul = DIR == 0 ? load_cell1(u, g, i - 1, j) : load_cell1(u, g, i, j - 1);
      ur = load_cell1(u, g, i, j);
    } else {
      ul = load_cell(u, k0 - step);
      ur = load_cell(u, k0);
    }
    set_normal_b<DIR>(ul, bn);
    set_normal_b<DIR>(ur, bn);
  }
  if (!recon_admissible(ul, gamma) || !recon_admissible(ur, gamma)) {
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    ul = St{nan, nan, nan, nan, nan, nan, nan, nan};
    ur = ul;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    out.L[c][k0] = comp(ul, c);
    out.R[c][k0] = comp(ur, c);
  }
}

template <int DIR, int ORDER, int MODE = 0>
__device__ __forceinline__ void b_reconstruct(const Grid& g, const StateP& u, const IfaceP& out,
                                              double gamma, const Ctl* ctl, int bx, int by,
                                              int* label = nullptr,
                                              FaceList defer = FaceList{}) {
  // dir 0: faces i in [0,nx] over all padded rows; dir 1: transposed.
  const int i = bx * blockDim.x + threadIdx.x - (DIR == 1 ? g.ng : 0);
  const int j = by * blockDim.y + threadIdx.y - (DIR == 0 ? g.ng : 0);
  const bool valid = !(DIR == 0 ? (i > g.nx || j >= g.ny + g.ng) : (i >= g.nx + g.ng || j > g.ny));
  if (ctl->status & ~kStatusDone) return;  // uniform: no kernel of a step writes it mid-launch
  if constexpr (MODE == 0 && ORDER >= 5) {
    // the characteristic path, warp-cooperative (threadIdx.y = warp)
    extern __shared__ double dsm[];
    mp_faces_warp<DIR, ORDER>(g, u, out, gamma, i, j, valid, dsm + threadIdx.y * kWarpReconDoubles);
    return;
  }
  if (!valid) return;
  recon_face<DIR, ORDER, MODE>(g, u, out, gamma, i, j, label, defer);
}

template <int DIR, int ORDER>
__global__ void __launch_bounds__(128, 4) k_reconstruct(Grid g, StateP u, IfaceP out, double gamma,
                                                        const Ctl* ctl) {
  b_reconstruct<DIR, ORDER>(g, u, out, gamma, ctl, blockIdx.x, blockIdx.y);
}

// Limiter labels of the cells (training data of the indicator): the
// departure of the limited states (literal = 0) or whether the limiter fired
// (literal = 1).
template <int DIR, int ORDER>
__global__ void __launch_bounds__(128) k_reconstruct_label(Grid g, StateP u, IfaceP out,
                                                           double gamma, const Ctl* ctl,
                                                           int* label, int literal) {
  if (literal)
    b_reconstruct<DIR, ORDER, 3>(g, u, out, gamma, ctl, blockIdx.x, blockIdx.y, label);
  else
    b_reconstruct<DIR, ORDER, 1>(g, u, out, gamma, ctl, blockIdx.x, blockIdx.y, label);
}

// Learned mode, pass 1: every face by the unlimited component-wise path
// (inadmissible ones deferred to pass 2).  Memory-latency bound: at 64
// registers and eight blocks per SM it ran 17% faster than at 94 and five.
// mp_pair_lin from a shared-memory tile: component v's stencil cell t at
// tile[v pc + pos + t tstep]; the same operations in the same order.
template <int DIR, int H>
__device__ __forceinline__ void mp_pair_lin_tile(const double* tile, int pc, int pos, int tstep,
                                                 St& ul, St& ur) {
  constexpr int S = 2 * H + 2, W = 2 * H + 1;
  double dl[8], dr[8], cv[8];
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const double* a = tile + v * pc + pos;
    const double c = 0.5 * a[H * tstep] + 0.5 * a[(H + 1) * tstep];
    cv[v] = c;
    if (v == 5) continue;  // the normal field is not reconstructed
    double w[S];
#pragma unroll
    for (int t = 0; t < S; ++t) w[t] = a[t * tstep] - c;
    dl[v] = mp_interp_plain<W>(w);
    double wr[W];
#pragma unroll
    for (int t = 0; t < W; ++t) wr[t] = w[W - t];
    dr[v] = mp_interp_plain<W>(wr);
  }
  const St sl{cv[0] + dl[0], cv[1] + dl[1], cv[2] + dl[2], cv[3] + dl[3],
              cv[4] + dl[4], cv[5],         cv[6] + dl[6], cv[7] + dl[7]};
  const St sr{cv[0] + dr[0], cv[1] + dr[1], cv[2] + dr[2], cv[3] + dr[3],
              cv[4] + dr[4], cv[5],         cv[6] + dr[6], cv[7] + dr[7]};
  ul = rot<DIR>(sl);
  ur = rot<DIR>(sr);
}

// The block's stencil cells (canonical components) are staged in shared
// memory once, each read by up to 2H + 2 faces (5.7 -> 5.0 ms of component-wise
// and listed passes per learned rotor 4096^2 MP7 step, the state
// bit-identical).  Every stencil cell of a valid face lies inside the padded
// grid, so the staged values are the ones the per-face loads read.
template <int DIR, int ORDER>
__global__ void __launch_bounds__(128, 8) k_reconstruct_lin(Grid g, StateP u, IfaceP out,
                                                         double gamma, const Ctl* ctl,
                                                         FaceList defer) {
  constexpr int H = ORDER == 5 ? 2 : 3, S = 2 * H + 2;
  constexpr int TW = DIR == 0 ? kBX + S - 1 : kBX;  // staged columns
  constexpr int TH = DIR == 0 ? 4 : 4 + S - 1;      // staged rows
  constexpr int PC = TW * TH;
  __shared__ double tile[8 * PC];
  if (ctl->status & ~kStatusDone) return;  // uniform: no kernel of a step writes it mid-launch
  const int i0 = blockIdx.x * kBX - (DIR == 1 ? g.ng : 0);
  const int j0 = blockIdx.y * 4 - (DIR == 0 ? g.ng : 0);
  const int ci0 = DIR == 0 ? i0 - 1 - H : i0, cj0 = DIR == 0 ? j0 : j0 - 1 - H;
  const int tid = threadIdx.y * kBX + threadIdx.x;
  for (int e = tid; e < PC; e += kBX * 4) {
    const int r = e / TW, c = e - r * TW;
    const int ci = ci0 + c, cj = cj0 + r;
    const bool in = ci >= -g.ng && ci < g.nx + g.ng && cj >= -g.ng && cj < g.ny + g.ng;
    const long long k = in ? g.idx(ci, cj) : 0;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const double* a = v == 0 ? u.c[0]
                        : v == 1 ? (DIR == 0 ? u.c[1] : u.c[2])
                        : v == 2 ? (DIR == 0 ? u.c[2] : u.c[1])
                        : v == 3 ? u.c[3]
                        : v == 4 ? u.c[4]
                        : v == 5 ? (DIR == 0 ? u.bxc : u.byc)
                        : v == 6 ? (DIR == 0 ? u.byc : u.bxc)
                                 : u.c[7];
      tile[v * PC + e] = in ? __ldg(a + k) : 0.0;
    }
  }
  __syncthreads();
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  const bool valid = !(DIR == 0 ? (i > g.nx || j >= g.ny + g.ng) : (i >= g.nx + g.ng || j > g.ny));
  if (!valid) return;
  const long long k0 = g.idx(i, j);
  const long long step = DIR == 0 ? 1 : g.pitch;
  St ul, ur;
  mp_pair_lin_tile<DIR, H>(tile, PC, threadIdx.y * TW + threadIdx.x, DIR == 0 ? 1 : TW, ul, ur);
  if (!recon_admissible(ul, gamma) || !recon_admissible(ur, gamma)) {
    if (!defer.flag[k0 - step] && !defer.flag[k0]) defer.list[atomicAdd(defer.count, 1)] = int(k0);
    return;
  }
  finish_face<DIR, ORDER, 2>(g, u, out, gamma, i, j, k0, step, ul, ur);
}

// Learned mode, pass 2: the listed faces (padded linear index of the face's
// high cell) by the full characteristic path; the count is read on the device.
// Warps take 32 consecutive list entries at a time.
template <int DIR, int ORDER>
__device__ __forceinline__ void b_reconstruct_list(const Grid& g, const StateP& u,
                                                   const IfaceP& out, double gamma,
                                                   const int* list, int n) {
  extern __shared__ double dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ws = dsm + warp * kWarpReconDoubles;
  for (int base = (blockIdx.x * kReconWarps + warp) * 32; base < n;
       base += gridDim.x * kReconWarps * 32) {
    const int t = base + lane;
    const bool valid = t < n;
    int i = 0, j = 0;
    if (valid) {
      const int k = list[t];
      i = k % g.pitch - g.ng;
      j = k / g.pitch - g.ng;
    }
    mp_faces_warp<DIR, ORDER>(g, u, out, gamma, i, j, valid, ws);
  }
}

template <int DIR, int ORDER>
__global__ void __launch_bounds__(128, 4) k_reconstruct_list(Grid g, StateP u, IfaceP out,
                                                             double gamma, const Ctl* ctl,
                                                             const int* list, const int* count) {
  if (ctl->status & ~kStatusDone) return;
  b_reconstruct_list<DIR, ORDER>(g, u, out, gamma, list, *count);
}

// Faces whose either cell is flagged, appended to the x and y lists in
// warp-aggregated order; padded cells are scanned row-major.
__global__ void k_face_lists(Grid g, const unsigned char* flag, int* xlist, int* ylist,
                             int* counts) {
  const long long n = g.size();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const unsigned lane = threadIdx.x & 31;
  bool nx_ = false, ny_ = false;
  int k = 0;
  if (t < n) {
    k = int(t);
    const int i = int(t % g.pitch) - g.ng, j = int(t / g.pitch) - g.ng;
    if (i >= 0 && i <= g.nx && j < g.ny + g.ng) nx_ = (flag[t] | flag[t - 1]) != 0;
    if (j >= 0 && j <= g.ny && i < g.nx + g.ng) ny_ = (flag[t] | flag[t - g.pitch]) != 0;
  }
  const unsigned bx_ = __ballot_sync(0xffffffffu, nx_), by_ = __ballot_sync(0xffffffffu, ny_);
  int basex = 0, basey = 0;
  if (lane == 0) {
    if (bx_) basex = atomicAdd(&counts[0], __popc(bx_));
    if (by_) basey = atomicAdd(&counts[1], __popc(by_));
  }
  basex = __shfl_sync(0xffffffffu, basex, 0);
  basey = __shfl_sync(0xffffffffu, basey, 0);
  const unsigned below = (1u << lane) - 1u;
  if (nx_) xlist[basex + __popc(bx_ & below)] = k;
  if (ny_) ylist[basey + __popc(by_ & below)] = k;
}


}  // namespace

// ===========================================================================
// Face flux (mhd_riemann.hip:53-136, mhd_face_quadrature.hpp:114-273) with
// the CT face EMF of the same solve (mhd_ct.hip:330-359) and the CFL face
// signal speed (mhd_reduce.hip:254-416).
// ===========================================================================
namespace {

struct Spd {
  double v, f;
};

// One side's |v_n| and fast speed (mhd_reduce.hip:254-325), with one
// reciprocal of rho.  The discriminant is formed as (a^2 - b^2)^2 + 4 a^2 b_t^2,
// which equals the reference's (a^2 + b^2)^2 - 4 a^2 b_n^2 but has no
// cancellation: where the reference's rounding is amplified to sqrt(eps) (a
// degenerate fan, a == b_n with b_t == 0) this form stays accurate to a few
// ulps, and elsewhere both agree to rounding.
template <int DIR>
__device__ Spd speed_parts(const St& s, double gamma) {
  if (!(isfinite(s.rho) && s.rho > 0.0 && isfinite(s.mx) && isfinite(s.my) &&
        isfinite(s.mz) && isfinite(s.E) && isfinite(s.bx) && isfinite(s.by) && isfinite(s.bz)))
    return Spd{kInf, kInf};
  const double ir = 1.0 / s.rho;
  const double p = pressure_f(s, gamma, ir);
  if (!(isfinite(p) && p > 0.0)) return Spd{kInf, kInf};
  const double bn = DIR == 0 ? s.bx : s.by, b1 = DIR == 0 ? s.by : s.bx;
  const double a2 = gamma * p * ir;
  const double bn2 = bn * bn * ir;
  const double bt2 = (b1 * b1 + s.bz * s.bz) * ir;
  const double d = a2 - (bn2 + bt2);
  const double disc = d * d + 4.0 * a2 * bt2;
  const double fast = sqrt(0.5 * ((a2 + bn2 + bt2) + sqrt(disc)));
  const double vel = fabs(DIR == 0 ? s.mx : s.my) * ir;
  if (!(isfinite(vel) && isfinite(fast))) return Spd{kInf, kInf};
  return Spd{vel, fast};
}

// Weighted face rate 0.5*alpha/h of one Riemann problem (mhd_reduce.hip:331-383).
template <int DIR, int ORDER>
__device__ __forceinline__ double face_rate(const St& l, const St& r, double gamma, double h) {
  const Spd a = speed_parts<DIR>(l, gamma), b = speed_parts<DIR>(r, gamma);
  const double rate = ORDER <= 1 ? fmax(a.v + a.f, b.v + b.f) : fmax(a.v, b.v) + fmax(a.f, b.f);
  if (!(isfinite(rate) && rate >= 0.0)) return kInf;
  return div_by(rate * 0.5, h, pow2_recip(h));
}

__device__ __forceinline__ St iface(const IfaceP& v, long long k, bool left) {
  if (left)
    return St{__ldg(v.L[0] + k), __ldg(v.L[1] + k), __ldg(v.L[2] + k), __ldg(v.L[3] + k),
              __ldg(v.L[4] + k), __ldg(v.L[5] + k), __ldg(v.L[6] + k), __ldg(v.L[7] + k)};
  return St{__ldg(v.R[0] + k), __ldg(v.R[1] + k), __ldg(v.R[2] + k), __ldg(v.R[3] + k),
            __ldg(v.R[4] + k), __ldg(v.R[5] + k), __ldg(v.R[6] + k), __ldg(v.R[7] + k)};
}

template <int DIR, int ORDER>
__global__ void __launch_bounds__(128) k_face_flux(Grid g, IfaceP in, FluxP out, double* emf,
                                                   int* nj, double* spd, double gamma,
                                                   const Ctl* ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.nx || j > g.ny) return;
  if (ctl->status & ~kStatusDone) return;
  int si = i, sj = j;
  // The periodic high face repeats face 0's Riemann data bit for bit.
  if (DIR == 0 && i == g.nx && g.bc[0] == 0 && g.bc[1] == 0) si = 0;
  if (DIR == 1 && j == g.ny && g.bc[2] == 0 && g.bc[3] == 0) sj = 0;
  const long long k = g.idx(i, j), ks = g.idx(si, sj);
  const double h = DIR == 0 ? g.dx : g.dy;
  const St bl = iface(in, ks, true), br = iface(in, ks, false);
  Fx f;
  double rate = 0.0;
  constexpr bool kLF = ORDER <= 1;
  if (ORDER != 5 && ORDER != 7) {
    f = riemann<DIR>(bl, br, kLF, gamma);
    if (spd) rate = face_rate<DIR, ORDER>(bl, br, gamma, h);
  } else {
    constexpr int H = ORDER == 5 ? 2 : 3, N = 2 * H + 1, Q = ORDER == 5 ? 3 : 4;
    const long long ts = DIR == 0 ? g.pitch : 1;
    // Recover the Q Gauss-point states of both sides from N transverse face
    // averages (mhd_face_quadrature.hpp:114-142).
    double pl[Q][8], pr[Q][8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      double sa[N], sb[N];
#pragma unroll
      for (int t = 0; t < N; ++t) {
        sa[t] = __ldg(in.L[c] + ks + (t - H) * ts);
        sb[t] = __ldg(in.R[c] + ks + (t - H) * ts);
      }
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        pl[q][c] = point_value<ORDER>(q, sa);
        pr[q][c] = point_value<ORDER>(q, sb);
      }
    }
    bool ok = true;
    int first_bad = Q;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const St l{pl[q][0], pl[q][1], pl[q][2], pl[q][3], pl[q][4], pl[q][5], pl[q][6], pl[q][7]};
      const St r{pr[q][0], pr[q][1], pr[q][2], pr[q][3], pr[q][4], pr[q][5], pr[q][6], pr[q][7]};
      if (!point_admissible(l, gamma) || !point_admissible(r, gamma)) {
        ok = false;
        if (first_bad == Q) first_bad = q;
      }
    }
    if (spd) {
      rate = face_rate<DIR, ORDER>(bl, br, gamma, h);
      for (int q = 0; q < first_bad; ++q) {
        const St l{pl[q][0], pl[q][1], pl[q][2], pl[q][3], pl[q][4], pl[q][5], pl[q][6], pl[q][7]};
        const St r{pr[q][0], pr[q][1], pr[q][2], pr[q][3], pr[q][4], pr[q][5], pr[q][6], pr[q][7]};
        rate = fmax(rate, face_rate<DIR, ORDER>(l, r, gamma, h));
      }
    }
    if (!ok) {
      // A transverse polynomial may leave the admissible set: fall back to the
      // face-average problem (mhd_face_quadrature.hpp:234-239).
      f = riemann<DIR>(bl, br, kLF, gamma);
    } else {
      double fq[8][Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const St l{pl[q][0], pl[q][1], pl[q][2], pl[q][3], pl[q][4], pl[q][5], pl[q][6], pl[q][7]};
        const St r{pr[q][0], pr[q][1], pr[q][2], pr[q][3], pr[q][4], pr[q][5], pr[q][6], pr[q][7]};
        const Fx fl = riemann<DIR>(l, r, kLF, gamma);
        fq[0][q] = fl.rho; fq[1][q] = fl.mx; fq[2][q] = fl.my; fq[3][q] = fl.mz;
        fq[4][q] = fl.E;   fq[5][q] = fl.bx; fq[6][q] = fl.by; fq[7][q] = fl.bz;
      }
      f.rho = gauss_avg<ORDER>(fq[0]);
      f.mx = gauss_avg<ORDER>(fq[1]);
      f.my = gauss_avg<ORDER>(fq[2]);
      f.mz = gauss_avg<ORDER>(fq[3]);
      f.E = gauss_avg<ORDER>(fq[4]);
      f.bx = gauss_avg<ORDER>(fq[5]);
      f.by = gauss_avg<ORDER>(fq[6]);
      f.bz = gauss_avg<ORDER>(fq[7]);
    }
  }
  // out, emf and nj may each be absent (the per-kernel launch interface
  // asks for fluxes or for the CT face tables alone)
  if (out.f[0]) {
    out.f[0][k] = f.rho;
    out.f[1][k] = f.mx;
    out.f[2][k] = f.my;
    out.f[3][k] = f.mz;
    out.f[4][k] = f.E;
    out.f[5][k] = f.bx;
    out.f[6][k] = f.by;
    out.f[7][k] = f.bz;
  }
  // Directional Godunov E_z: F_x(By) = -Ez, F_y(Bx) = +Ez (mhd_ct.hip:126-133).
  if (emf) emf[k] = DIR == 0 ? -f.by : f.bx;
  if (spd) spd[k] = rate;
  if (!nj) return;
  // "No jump" proof of the complete point-recovered problem
  // (mhd_ct.hip:150-174); taps are mapped like every CT table read.
  constexpr int RH = ORDER >= 7 ? 3 : ORDER >= 5 ? 2 : 0;
  int proof = 1;
  for (int off = -RH; off <= RH && proof; ++off) {
    const int mi = face_index(DIR == 0 ? i : i + off, g.nx, g.bc[0], g.bc[1]);
    const int mj = face_index(DIR == 0 ? j + off : j, g.ny, g.bc[2], g.bc[3]);
    if (!in_pad(g, mi, mj)) {
      proof = 0;
      break;
    }
    const long long km = g.idx(mi, mj);
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (!(in.L[c][km] == in.R[c][km])) proof = 0;
  }
  nj[k] = proof;
}

}  // namespace

// ---------------------------------------------------------------------------
// MP5/MP7 face flux with one lane per Gauss point: a group of Q lanes owns a
// face (Q = 3 at MP5, 4 at MP7).  The interface states of a face tile (8 x 4
// at MP7, 8 x 5 at MP5) and its transverse halo are staged in shared memory,
// so each stencil row is read from L2 once per tile instead of once per face
// row (2.8x fewer for x faces, 4x for y faces at MP7).  At MP7 the
// transverse recovery is split by component: lane q forms components q,
// q + 4, ... at every Gauss point of its face (each stencil column read
// once, and the constant-stencil shortcut, which decides the same for every
// point, tested once per component) into the face's point rows in shared
// memory, from which each lane takes its own point's 16 components as
// 16-byte pairs.  Each lane solves its point's Riemann problem, the group
// votes on admissibility, and the point fluxes go back through the same
// rows, where lane q forms and stores the Gauss sums of components q, q + 4
// (rotor 4096^2 MP7: face flux 27.6 -> 23.3 ms per step; Orszag-Tang 2048^2
// MP7: 10.8 -> 10.4).  At MP5 each lane recovers its own point (below).
// Same sums in the same node order as k_face_flux; the compiler's fused
// multiply-adds may pair differently, a rounding-level difference.  128 threads
// (smaller blocks than 16 x 4 measured 3-5% faster at MP7: a block waiting
// at the staging barrier holds fewer warps).
// ---------------------------------------------------------------------------
namespace {

constexpr int kFqTX = 8, kFqTY = 4;
// One lane per Gauss point: groups of 4 lanes (MP7, 8 faces per warp, 8 x 4
// face tiles) or 3 lanes (MP5, 10 faces per warp with two lanes idle, 8 x 5
// tiles); four warps per block either way.
constexpr int kFqThreads = 4 * kFqTX * kFqTY;
template <int ORDER>
constexpr int fq_ty() { return ORDER == 5 ? 5 : 4; }
// 96 registers (ptxas keeps a few values of the HLLD tail on the stack):
// five 128-thread blocks per SM measured 8-11% faster than four at 128
// registers (six spill more and lose it again).
constexpr int kFqBlocksPerSm = 5;
// Shared-memory strides in doubles.  A component plane of the tile is padded
// to 4 mod 16 doubles, so that the lanes of a group (components 4 apart of
// one cell) and the neighbouring groups (neighbouring cells) read distinct
// banks; a point row is 16 components + 2 (16-byte aligned), a face's rows
// are Q rows + 4.
constexpr int fq_plane(int cells) { return cells + ((4 - cells % 16) + 16) % 16; }
constexpr int kFqRow = 18;
template <int ORDER>
constexpr int fq_face() { return (ORDER == 5 ? 3 : 4) * kFqRow + 4; }

// Per-point recovery (MP5): each lane forms all 16 components of its own
// Gauss point from the staged tile, and the group gathers the point fluxes
// by shuffles.  With three lanes per face the component split below leaves
// a lane with six components against five and measured 8% slower on
// Orszag-Tang 2048^2 MP5 (face flux 9.1 -> 9.8 ms per step).
template <int DIR, int ORDER, int TX = kFqTX>
__device__ __forceinline__ void b_face_flux_pt(const Grid& g, const IfaceP& in, const FluxP& out,
                                               double* emf, int* nj, double* spd, double gamma,
                                               const Ctl* ctl, int bx, int by) {
  constexpr int H = ORDER == 5 ? 2 : 3, N = 2 * H + 1, Q = ORDER == 5 ? 3 : 4;
  constexpr int FPW = 32 / Q, TY = fq_ty<ORDER>();         // faces per warp, tile rows
  static_assert(4 * FPW == TX * TY, "four warps cover the face tile");
  constexpr int TR = DIR == 0 ? TY + 2 * H : TY;          // tile rows (j)
  constexpr int TC = DIR == 0 ? TX : TX + 2 * H;          // tile columns (i)
  __shared__ double tile[16][TR][TC];
  __shared__ unsigned char same[TR][TC];  // staged and L == R in every component
  if (ctl->status) return;  // uniform over the block
  const int i0 = bx * TX, j0 = by * TY;
  const bool perx = g.bc[0] == 0 && g.bc[1] == 0, pery = g.bc[2] == 0 && g.bc[3] == 0;
  for (int e = threadIdx.x; e < TR * TC; e += blockDim.x) {
    const int row = e / TC, col = e - row * TC;
    int fi, fj;
    bool valid;
    if (DIR == 0) {
      const int ii = i0 + col;
      fi = (ii == g.nx && perx) ? 0 : ii;
      fj = j0 - H + row;
      valid = ii <= g.nx && fj >= -g.ng && fj < g.ny + g.ng;
    } else {
      const int jj = j0 + row;
      fj = (jj == g.ny && pery) ? 0 : jj;
      fi = i0 - H + col;
      valid = jj <= g.ny && fi >= -g.ng && fi < g.nx + g.ng;
    }
    const long long kk = valid ? g.idx(fi, fj) : 0;
    bool eq = valid;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double a = valid ? __ldg(in.L[c] + kk) : 0.0;
      const double b = valid ? __ldg(in.R[c] + kk) : 0.0;
      tile[c][row][col] = a;
      tile[8 + c][row][col] = b;
      eq = eq && a == b;
    }
    same[row][col] = eq;
  }
  __syncthreads();
  constexpr bool kLF = false;
  const int wl = threadIdx.x & 31;
  if (wl >= FPW * Q) return;  // the lanes no group uses (MP5)
  const int lane = wl % Q, base = wl - lane;
  const unsigned gmask = ((1u << Q) - 1u) << base;
  const int face = (threadIdx.x >> 5) * FPW + wl / Q;
  const int fx = face % TX, fy = face / TX;
  const int i = i0 + fx, j = j0 + fy;
  if (i > g.nx || j > g.ny) return;  // whole groups leave together
  const long long k = g.idx(i, j);
  const double h = DIR == 0 ? g.dx : g.dy;
  // tile coordinates of stencil tap t (t = H is the face itself)
  auto tr = [&](int t) { return DIR == 0 ? fy + t : fy; };
  auto tcl = [&](int t) { return DIR == 0 ? fx : fx + t; };
  St l{}, r{};
  double irl = 1.0, irr = 1.0;
  bool ok = true;
  {
    double w[N];
#pragma unroll
    for (int t = 0; t < N; ++t) w[t] = point_w<ORDER>(lane, t);
    double pl[8], pr[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      double sa[N], sb[N];
#pragma unroll
      for (int t = 0; t < N; ++t) {
        sa[t] = tile[c][tr(t)][tcl(t)];
        sb[t] = tile[8 + c][tr(t)][tcl(t)];
      }
      pl[c] = wsum<N>(w, sa);
      pr[c] = wsum<N>(w, sb);
    }
    l = St{pl[0], pl[1], pl[2], pl[3], pl[4], pl[5], pl[6], pl[7]};
    r = St{pr[0], pr[1], pr[2], pr[3], pr[4], pr[5], pr[6], pr[7]};
    irl = 1.0 / l.rho;
    irr = 1.0 / r.rho;
    ok = point_admissible_ir(l, gamma, irl) && point_admissible_ir(r, gamma, irr);
  }
  auto centre = [&](bool left) {
    const int o = left ? 0 : 8, rr = tr(H), cc = tcl(H);
    return St{tile[o][rr][cc],     tile[o + 1][rr][cc], tile[o + 2][rr][cc], tile[o + 3][rr][cc],
              tile[o + 4][rr][cc], tile[o + 5][rr][cc], tile[o + 6][rr][cc], tile[o + 7][rr][cc]};
  };
  const unsigned bad = (__ballot_sync(gmask, !ok) >> base) & ((1u << Q) - 1u);
  const bool group_ok = bad == 0;
  const int first_bad = bad ? __ffs(bad) - 1 : Q;
  double rate = 0.0;
  if (spd) {
    if (lane == 0) rate = face_rate<DIR, ORDER>(centre(true), centre(false), gamma, h);
    if (lane < first_bad) rate = fmax(rate, face_rate<DIR, ORDER>(l, r, gamma, h));
  }
  const bool solve = group_ok || lane == 0;
  if (!group_ok) {
    l = centre(true);
    r = centre(false);
    irl = 1.0 / l.rho;
    irr = 1.0 / r.rho;
  }
  double fv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (solve) {
    const Fx f = riemann<DIR>(l, r, kLF, gamma, irl, irr);
    fv[0] = f.rho; fv[1] = f.mx; fv[2] = f.my; fv[3] = f.mz;
    fv[4] = f.E;   fv[5] = f.bx; fv[6] = f.by; fv[7] = f.bz;
  }
  double res[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    if (group_ok) {
      double sq[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) sq[q] = __shfl_sync(gmask, fv[c], base + q);
      res[c] = gauss_avg<ORDER>(sq);
    } else {
      res[c] = __shfl_sync(gmask, fv[c], base);
    }
  }
  // out, emf and nj may each be absent (the per-kernel launch interface
  // asks for fluxes or for the CT face tables alone); the stores are split
  // over the group (component c by lane c mod Q)
  if (out.f[0]) {
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (c % Q == lane) out.f[c][k] = res[c];
  }
  if (lane == 0 && emf) emf[k] = DIR == 0 ? -res[6] : res[5];
  if (spd) {
    double m = rate;
#pragma unroll
    for (int q = 0; q < Q; ++q) m = fmax(m, __shfl_sync(gmask, rate, base + q));
    if (lane == 0) spd[k] = m;
  }
  if (!nj) return;  // uniform over the block
  // no-jump proof over the 2H+1 transverse taps (mapped like every CT table
  // read), split across the group.  A tap whose mapped face is the one staged
  // in its tile slot reads the staged comparison; the others read memory.
  int proof = 1;
  for (int off = lane - H; off <= H; off += Q) {
    const int mi = face_index(DIR == 0 ? i : i + off, g.nx, g.bc[0], g.bc[1]);
    const int mj = face_index(DIR == 0 ? j + off : j, g.ny, g.bc[2], g.bc[3]);
    const int ti = DIR == 0 ? ((i == g.nx && perx) ? 0 : i) : i + off;
    const int tj = DIR == 0 ? j + off : ((j == g.ny && pery) ? 0 : j);
    if (mi == ti && mj == tj) {
      if (!same[tr(off + H)][tcl(off + H)]) proof = 0;
      continue;
    }
    if (!in_pad(g, mi, mj)) {
      proof = 0;
      break;
    }
    const long long km = g.idx(mi, mj);
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (!(in.L[c][km] == in.R[c][km])) proof = 0;
  }
  const unsigned nproof = (__ballot_sync(gmask, proof == 0) >> base) & ((1u << Q) - 1u);
  if (lane == 0) nj[k] = nproof == 0 ? 1 : 0;
}

// Component-split recovery (MP7), as described above.
template <int DIR, int ORDER, int TX = kFqTX>
__device__ __forceinline__ void b_face_flux_cs(const Grid& g, const IfaceP& in, const FluxP& out,
                                               double* emf, int* nj, double* spd, double gamma,
                                               const Ctl* ctl, int bx, int by) {
  constexpr int H = ORDER == 5 ? 2 : 3, N = 2 * H + 1, Q = ORDER == 5 ? 3 : 4;
  constexpr int FPW = 32 / Q, TY = fq_ty<ORDER>();         // faces per warp, tile rows
  static_assert(4 * FPW == TX * TY, "four warps cover the face tile");
  constexpr int TR = DIR == 0 ? TY + 2 * H : TY;          // tile rows (j)
  constexpr int TC = DIR == 0 ? TX : TX + 2 * H;          // tile columns (i)
  constexpr int PS = fq_plane(TR * TC), FS = fq_face<ORDER>();
  __shared__ double tile[16 * PS];             // component c of slot (row, col): c PS + row TC + col
  __shared__ unsigned char same[TR][TC];       // staged and L == R in every component
  __shared__ __align__(16) double pts[4 * FPW * FS];  // per face: Q point rows
  if (ctl->status) return;  // uniform over the block
  const int i0 = bx * TX, j0 = by * TY;
  const bool perx = g.bc[0] == 0 && g.bc[1] == 0, pery = g.bc[2] == 0 && g.bc[3] == 0;
  for (int e = threadIdx.x; e < TR * TC; e += blockDim.x) {
    const int row = e / TC, col = e - row * TC;
    int fi, fj;
    bool valid;
    if (DIR == 0) {
      const int ii = i0 + col;
      fi = (ii == g.nx && perx) ? 0 : ii;
      fj = j0 - H + row;
      valid = ii <= g.nx && fj >= -g.ng && fj < g.ny + g.ng;
    } else {
      const int jj = j0 + row;
      fj = (jj == g.ny && pery) ? 0 : jj;
      fi = i0 - H + col;
      valid = jj <= g.ny && fi >= -g.ng && fi < g.nx + g.ng;
    }
    const long long kk = valid ? g.idx(fi, fj) : 0;
    bool eq = valid;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double a = valid ? __ldg(in.L[c] + kk) : 0.0;
      const double b = valid ? __ldg(in.R[c] + kk) : 0.0;
      tile[c * PS + e] = a;
      tile[(8 + c) * PS + e] = b;
      eq = eq && a == b;
    }
    same[row][col] = eq;
  }
  __syncthreads();
  constexpr bool kLF = false;
  const int wl = threadIdx.x & 31;
  if (wl >= FPW * Q) return;  // the lanes no group uses (MP5)
  const int lane = wl % Q, base = wl - lane;
  const unsigned gmask = ((1u << Q) - 1u) << base;
  const int face = (threadIdx.x >> 5) * FPW + wl / Q;
  const int fx = face % TX, fy = face / TX;
  const int i = i0 + fx, j = j0 + fy;
  if (i > g.nx || j > g.ny) return;  // whole groups leave together
  const long long k = g.idx(i, j);
  const double h = DIR == 0 ? g.dx : g.dy;
  // tile slot of stencil tap t (t = H is the face itself)
  auto slot = [&](int t) { return DIR == 0 ? (fy + t) * TC + fx : fy * TC + fx + t; };
  double* const fp = pts + face * FS;  // this face's point rows
  // point values of components lane, lane + Q, ... at the Q Gauss nodes
#pragma unroll
  for (int m = 0; m < (16 + Q - 1) / Q; ++m) {
    const int c = lane + Q * m;
    if (c < 16) {
      double s[N], v[Q];
#pragma unroll
      for (int t = 0; t < N; ++t) s[t] = tile[c * PS + slot(t)];
      point_values<ORDER>(s, v);
#pragma unroll
      for (int p = 0; p < Q; ++p) fp[p * kFqRow + c] = v[p];
    }
  }
  __syncwarp(gmask);
  St l, r;
  {
    const double2* row = reinterpret_cast<const double2*>(fp + lane * kFqRow);
    const double2 a0 = row[0], a1 = row[1], a2 = row[2], a3 = row[3];
    const double2 b0 = row[4], b1 = row[5], b2 = row[6], b3 = row[7];
    l = St{a0.x, a0.y, a1.x, a1.y, a2.x, a2.y, a3.x, a3.y};
    r = St{b0.x, b0.y, b1.x, b1.y, b2.x, b2.y, b3.x, b3.y};
  }
  double irl = 1.0 / l.rho, irr = 1.0 / r.rho;
  const bool ok = point_admissible_ir(l, gamma, irl) && point_admissible_ir(r, gamma, irr);
  auto centre = [&](bool left) {
    const int o = left ? 0 : 8, sc = slot(H);
    return St{tile[o * PS + sc],       tile[(o + 1) * PS + sc], tile[(o + 2) * PS + sc],
              tile[(o + 3) * PS + sc], tile[(o + 4) * PS + sc], tile[(o + 5) * PS + sc],
              tile[(o + 6) * PS + sc], tile[(o + 7) * PS + sc]};
  };
  const unsigned bad = (__ballot_sync(gmask, !ok) >> base) & ((1u << Q) - 1u);
  const bool group_ok = bad == 0;
  const int first_bad = bad ? __ffs(bad) - 1 : Q;
  double rate = 0.0;
  if (spd) {
    if (lane == 0) rate = face_rate<DIR, ORDER>(centre(true), centre(false), gamma, h);
    if (lane < first_bad) rate = fmax(rate, face_rate<DIR, ORDER>(l, r, gamma, h));
  }
  const bool solve = group_ok || lane == 0;
  if (!group_ok) {
    l = centre(true);
    r = centre(false);
    irl = 1.0 / l.rho;
    irr = 1.0 / r.rho;
  }
  double fv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (solve) {
    const Fx f = riemann<DIR>(l, r, kLF, gamma, irl, irr);
    fv[0] = f.rho; fv[1] = f.mx; fv[2] = f.my; fv[3] = f.mz;
    fv[4] = f.E;   fv[5] = f.bx; fv[6] = f.by; fv[7] = f.bz;
  }
  // the point fluxes replace the lane's own point row (no other lane reads
  // it after the exchange above)
  {
    double2* row = reinterpret_cast<double2*>(fp + lane * kFqRow);
    row[0] = make_double2(fv[0], fv[1]);
    row[1] = make_double2(fv[2], fv[3]);
    row[2] = make_double2(fv[4], fv[5]);
    row[3] = make_double2(fv[6], fv[7]);
  }
  __syncwarp(gmask);
  // Gauss sums of components lane, lane + Q, ... in node order (or lane 0's
  // single solve at the face state when a point was not admissible)
  constexpr int RC = (8 + Q - 1) / Q;
  double res[RC];
#pragma unroll
  for (int m = 0; m < RC; ++m) {
    const int c = lane + Q * m;
    res[m] = 0.0;
    if (c < 8) {
      if (group_ok) {
        double sq[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) sq[q] = fp[q * kFqRow + c];
        res[m] = gauss_avg<ORDER>(sq);
      } else {
        res[m] = fp[c];
      }
    }
  }
  // out, emf and nj may each be absent (the per-kernel launch interface
  // asks for fluxes or for the CT face tables alone)
  if (out.f[0]) {
#pragma unroll
    for (int m = 0; m < RC; ++m)
      if (lane + Q * m < 8) out.f[lane + Q * m][k] = res[m];
  }
  // face E_z = -F(by) of an x face, F(bx) of a y face: the lane holding it
  constexpr int EC = DIR == 0 ? 6 : 5;
  if (emf && lane == EC % Q) emf[k] = DIR == 0 ? -res[EC / Q] : res[EC / Q];
  if (spd) {
    double m = rate;
#pragma unroll
    for (int q = 0; q < Q; ++q) m = fmax(m, __shfl_sync(gmask, rate, base + q));
    if (lane == 0) spd[k] = m;
  }
  if (!nj) return;  // uniform over the block
  // no-jump proof over the 2H+1 transverse taps (mapped like every CT table
  // read), split across the group.  A tap whose mapped face is the one staged
  // in its tile slot reads the staged comparison; the others read memory.
  int proof = 1;
  for (int off = lane - H; off <= H; off += Q) {
    const int mi = face_index(DIR == 0 ? i : i + off, g.nx, g.bc[0], g.bc[1]);
    const int mj = face_index(DIR == 0 ? j + off : j, g.ny, g.bc[2], g.bc[3]);
    const int ti = DIR == 0 ? ((i == g.nx && perx) ? 0 : i) : i + off;
    const int tj = DIR == 0 ? j + off : ((j == g.ny && pery) ? 0 : j);
    if (mi == ti && mj == tj) {
      const int sl = slot(off + H);
      if (!same[sl / TC][sl % TC]) proof = 0;
      continue;
    }
    if (!in_pad(g, mi, mj)) {
      proof = 0;
      break;
    }
    const long long km = g.idx(mi, mj);
#pragma unroll
    for (int c = 0; c < 8; ++c)
      if (!(in.L[c][km] == in.R[c][km])) proof = 0;
  }
  const unsigned nproof = (__ballot_sync(gmask, proof == 0) >> base) & ((1u << Q) - 1u);
  if (lane == 0) nj[k] = nproof == 0 ? 1 : 0;
}

// TX: faces per tile row; the block is four warps of 32 / Q groups each.
template <int DIR, int ORDER, int TX = kFqTX>
__device__ __forceinline__ void b_face_flux_qs(const Grid& g, const IfaceP& in, const FluxP& out,
                                               double* emf, int* nj, double* spd, double gamma,
                                               const Ctl* ctl, int bx, int by) {
  if constexpr (ORDER == 7)
    b_face_flux_cs<DIR, ORDER, TX>(g, in, out, emf, nj, spd, gamma, ctl, bx, by);
  else
    b_face_flux_pt<DIR, ORDER, TX>(g, in, out, emf, nj, spd, gamma, ctl, bx, by);
}

template <int DIR, int ORDER>
__global__ void __launch_bounds__(kFqThreads, kFqBlocksPerSm)
    k_face_flux_qs(Grid g, IfaceP in, FluxP out, double* emf, int* nj, double* spd, double gamma,
                   const Ctl* ctl) {
  b_face_flux_qs<DIR, ORDER, kFqTX>(g, in, out, emf, nj, spd, gamma, ctl, blockIdx.x,
                                          blockIdx.y);
}

}  // namespace

// ===========================================================================
// Constrained transport and the stage update
// ===========================================================================
namespace {

// E_z = -(v x B)_z (mhd_ct.hip:408-417, zero background)
// E_z = -(v x B)_z from the state and its 1/rho (one reciprocal shared with
// the point's admissibility test instead of a division per velocity
// component: a rounding-level difference)
__device__ __forceinline__ double physical_ez_ir(const St& s, double ir) {
  const double vx = s.mx * ir, vy = s.my * ir;
  return __dadd_rn(__dmul_rn(vy, s.bx), __dmul_rn(vx, -s.by));
}
__device__ __forceinline__ double physical_ez(const St& s) { return physical_ez_ir(s, 1.0 / s.rho); }

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Cell-average E_z by tensor Gauss quadrature of recovered point states
// (mhd_ct.hip:457-629); on stage 0 also the CFL max-reduction over cells
// (mhd_reduce.hip:418-501): warp shuffles, one atomic per block.
template <int ORDER>
__global__ void __launch_bounds__(128) k_cell_emf(Grid g, StateP u, double* cell_ez,
                                                  const double* xs, const double* ys,
                                                  int cfl_reduce, double gamma, Ctl* ctl) {
  __shared__ int s_stop;
  __shared__ double s_max[4];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  if (tid == 0) s_stop = ctl->status;
  __syncthreads();
  if (s_stop) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const bool phx = g.bc[1] != 0, phy = g.bc[3] != 0;
  if (i <= g.nx && j <= g.ny && !((i == g.nx && !phx) || (j == g.ny && !phy))) {
    const long long k = g.idx(i, j);
    const St c0 = ORDER <= 1 ? load_cell1(u, g, i, j) : load_cell(u, k);
    double e = physical_ez(c0);
    constexpr int H = ORDER >= 7 ? 3 : 2, N = 2 * H + 1, Q = ORDER >= 7 ? 4 : 3;
    if ((ORDER == 5 || ORDER == 7) && i - H >= -g.ng && i + H <= g.nx + g.ng - 1 &&
        j - H >= -g.ng && j + H <= g.ny + g.ng - 1) {
      double pt[Q][Q];
      bool ok = true;
      const double* src[8] = {u.c[0], u.c[1], u.c[2], u.c[3], u.c[4], u.bxc, u.byc, u.c[7]};
      for (int qx = 0; qx < Q && ok; ++qx) {
        double rows[8][N];
#pragma unroll
        for (int c = 0; c < 8; ++c)
#pragma unroll
          for (int r = 0; r < N; ++r) {
            double s[N];
            const long long kr = k + (long long)(r - H) * g.pitch;
#pragma unroll
            for (int t = 0; t < N; ++t) s[t] = __ldg(src[c] + kr + (t - H));
            rows[c][r] = point_value<ORDER>(qx, s);
          }
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) {
          const St p{point_value<ORDER>(qy, rows[0]), point_value<ORDER>(qy, rows[1]),
                     point_value<ORDER>(qy, rows[2]), point_value<ORDER>(qy, rows[3]),
                     point_value<ORDER>(qy, rows[4]), point_value<ORDER>(qy, rows[5]),
                     point_value<ORDER>(qy, rows[6]), point_value<ORDER>(qy, rows[7])};
          const double ir = 1.0 / p.rho;
          if (!point_admissible_ir(p, gamma, ir)) ok = false;
          pt[qy][qx] = physical_ez_ir(p, ir);
        }
      }
      if (ok) {
        double row[Q];
#pragma unroll
        for (int qy = 0; qy < Q; ++qy) row[qy] = gauss_avg<ORDER>(pt[qy]);
        e = gauss_avg<ORDER>(row);
      }
    }
    cell_ez[k] = e;
  }
  if (!cfl_reduce) return;
  double local = 0.0;
  if (i < g.nx && j < g.ny && g.in_window(i, j)) {
    const long long k = g.idx(i, j);
    const double r = (xs[k] + xs[k + 1]) + (ys[k] + ys[k + g.pitch]);
    local = isfinite(r) ? fmax(0.0, r) : kInf;
  }
  local = warp_max(local);
  if ((tid & 31) == 0) s_max[tid >> 5] = local;
  __syncthreads();
  if (tid == 0) {
    double m = s_max[0];
    for (int w = 1; w < (int)(blockDim.x * blockDim.y + 31) / 32; ++w) m = fmax(m, s_max[w]);
    atomicMax(&ctl->max_rate, dbits(m));
  }
}

// Tiled form of k_cell_emf for MP5/MP7: a 16x16 tile of cells and its
// H-wide halo are staged in shared memory once; for each x-node the
// x-recovered rows of the tile (all 8 components) are formed once in shared
// memory and every cell then recovers its y-nodes from them.  Same sums in
// the same order as k_cell_emf.  A square tile recovers fewer halo rows per
// cell than 32x8 (22/16 against 14/8 at MP7).
constexpr int kCellTX = 16, kCellTY = 16;

// TMA staging of the tile: rows of kTmaBW doubles (192 bytes) starting one
// cell left of the stencil's first column, so that the innermost coordinate
// of every copy is even (16-byte aligned); planes of SY rows are multiples of
// 128 bytes at both orders.
constexpr int kTmaBW = 24;

template <int ORDER, bool TMA = false>
constexpr int cell_smem_doubles() {
  constexpr int H = ORDER == 7 ? 3 : 2, SY = kCellTY + 2 * H;
  // TMA: 16 more doubles so that the staged planes can start on 128 bytes
  return 8 * SY * (TMA ? kTmaBW : kCellTX + 2 * H) + 8 * SY * kCellTX + (TMA ? 16 : 0);
}

// 3-D tiled TMA load of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y,
                                            int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(tc::smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// TMA: the eight state planes of the tile come in by one TMA copy each
// (issued by one thread, completing on an mbarrier whose wait is bounded)
// from `map`, the register's 3-D tensor map; out-of-range cells are filled
// with zeros by the copy, as the plain staging does.
template <int ORDER, bool TMA = false>
__device__ __forceinline__ void b_cell_emf_s(const Grid& g, const StateP& u, double* cell_ez,
                                             const double* xs, const double* ys, int cfl_reduce,
                                             double gamma, Ctl* ctl, int bx, int by,
                                             const CUtensorMap* map = nullptr) {
  constexpr int H = ORDER == 7 ? 3 : 2, N = 2 * H + 1, Q = ORDER == 7 ? 4 : 3;
  constexpr int TX = kCellTX, TY = kCellTY, SX = TX + 2 * H, SY = TY + 2 * H;
  // row stride and column offset of the staged tile: S[c][r][x] is the
  // stencil cell (i0 - H + x, j0 - H + r) at S + (c * SY + r) * RS + XO + x
  constexpr int RS = TMA ? kTmaBW : SX, XO = TMA ? 1 : 0;
  static_assert(!TMA || (SX + XO <= kTmaBW && (SY * kTmaBW * 8) % 128 == 0), "TMA box");
  extern __shared__ __align__(128) double sm[];
  // TMA destinations start on 128 bytes; the offset is taken inside the
  // shared array, so that the compiler keeps shared-memory loads (a pointer
  // rounded as an integer is generic: the cell EMF phase took 7.6 instead
  // of 7.1 ms per rotor 4096^2 MP7 step)
  double* S = TMA ? sm + ((128u - (tc::smem_u32(sm) & 127u)) & 127u) / sizeof(double)
                  : sm;          // [8][SY][RS] staged state
  double* X = S + 8 * SY * RS;  // [8][SY][TX] x-recovered rows of one x-node
  __shared__ int s_stop;
  __shared__ double s_max[8];
  __shared__ uint64_t s_bar;
  const int tid = threadIdx.y * TX + threadIdx.x;
  if (tid == 0) s_stop = ctl->status;
  __syncthreads();
  if (s_stop) return;
  const int i0 = bx * TX, j0 = by * TY;
  const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
  if constexpr (TMA) {
    // padded coordinates: x0 = i0 - H + ng - XO is even because ng - H = 1
    // at both orders and i0 is a multiple of 16
    if (tid == 0) {
      tc::mbar_init(&s_bar, 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      mbar_expect_tx(&s_bar, uint32_t(8 * SY * kTmaBW * sizeof(double)));
      const int x0 = i0 - H + g.ng - XO, y0 = j0 - H + g.ng;
      constexpr int kZ[8] = {0, 1, 2, 3, 4, 8, 9, 7};  // rho..E, bxc, byc, bz
#pragma unroll
      for (int c = 0; c < 8; ++c) tma_load_3d(S + c * SY * kTmaBW, map, x0, y0, kZ[c], &s_bar);
    }
    __syncthreads();  // the barrier is initialised before anyone waits on it
    // one warp polls the mbarrier; the others sleep in the block barrier,
    // which also orders the landed tile before their reads
    bool arrived = true;
    if (tid < 32) arrived = tc::mbar_wait(&s_bar, 0);
    if (!__syncthreads_and(arrived ? 1 : 0)) {
      // the copies did not land in time: report it, give them a second
      // bounded wait so that none is still writing when the block exits
      if (tid == 0) {
        atomicOr(&ctl->status, kStatusWaitExpired);
        tc::mbar_wait(&s_bar, 0);
      }
      __syncthreads();
      return;
    }
  } else {
  // staging: one index computation per staged cell, its 8 components
  // loaded with the same offset
  for (int r = threadIdx.y; r < SY; r += TY) {
    for (int x = threadIdx.x; x < SX; x += TX) {
      const int ii = i0 - H + x, jj = j0 - H + r;
      const bool in = in_pad(g, ii, jj);
      const long long kk = in ? g.idx(ii, jj) : 0;
      double* dst = S + r * SX + x;
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double* src = c < 5 ? u.c[c] : c == 5 ? u.bxc : c == 6 ? u.byc : u.c[7];
        dst[c * SY * SX] = in ? __ldg(src + kk) : 0.0;
      }
    }
  }
  __syncthreads();
  }
  const bool phx = g.bc[1] != 0, phy = g.bc[3] != 0;
  const bool active =
      i <= g.nx && j <= g.ny && !((i == g.nx && !phx) || (j == g.ny && !phy));
  double pt[Q][Q];
  bool ok = true;
#pragma unroll
  for (int qx = 0; qx < Q; ++qx) {
    double wx[N];
#pragma unroll
    for (int t = 0; t < N; ++t) wx[t] = point_w<ORDER>(qx, t);
    // x-recovery of every staged row (component c, row r) at this x node:
    // task = (row t = c * SY + r, column pair p); the two outputs' N + 1
    // taps come in as 16-byte loads (the staged rows start on 16 bytes;
    // with XO = 1 the pair's taps start one double into the first load)
    static_assert(RS % 2 == 0 && TX % 2 == 0, "16-byte rows");
    constexpr int NL = (XO + N + 2) / 2;  // 16-byte loads per pair
    for (int tk = tid; tk < 8 * SY * (TX / 2); tk += TX * TY) {
      const int t = tk / (TX / 2), pr = tk - t * (TX / 2);
      const double2* row = reinterpret_cast<const double2*>(S + t * RS + 2 * pr);
      double v[2 * NL];
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const double2 d = row[q];
        v[2 * q] = d.x;
        v[2 * q + 1] = d.y;
      }
      double s0[N], s1[N];
#pragma unroll
      for (int q = 0; q < N; ++q) {
        s0[q] = v[XO + q];
        s1[q] = v[XO + 1 + q];
      }
      reinterpret_cast<double2*>(X + t * TX)[pr] = make_double2(wsum<N>(wx, s0), wsum<N>(wx, s1));
    }
    __syncthreads();
    if (active && ok) {
      double st[Q][8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        double smp[N];
#pragma unroll
        for (int t = 0; t < N; ++t) smp[t] = X[(c * SY + threadIdx.y + t) * TX + threadIdx.x];
        if constexpr (ORDER == 7) {
          // the constant-stencil test once for the four y-nodes
          double pv[Q];
          point_values<ORDER>(smp, pv);
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) st[qy][c] = pv[qy];
        } else {
#pragma unroll
          for (int qy = 0; qy < Q; ++qy) st[qy][c] = point_value<ORDER>(qy, smp);
        }
      }
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) {
        const St p{st[qy][0], st[qy][1], st[qy][2], st[qy][3],
                   st[qy][4], st[qy][5], st[qy][6], st[qy][7]};
        const double ir = 1.0 / p.rho;
        if (!point_admissible_ir(p, gamma, ir)) ok = false;
        pt[qy][qx] = physical_ez_ir(p, ir);
      }
    }
    __syncthreads();
  }
  if (active) {
    const long long k = g.idx(i, j);
    double e;
    if (ok) {
      double row[Q];
#pragma unroll
      for (int qy = 0; qy < Q; ++qy) row[qy] = gauss_avg<ORDER>(pt[qy]);
      e = gauss_avg<ORDER>(row);
    } else {
      e = physical_ez(load_cell(u, k));
    }
    cell_ez[k] = e;
  }
  if (!cfl_reduce) return;
  double local = 0.0;
  if (i < g.nx && j < g.ny && g.in_window(i, j)) {
    const long long k = g.idx(i, j);
    const double r = (xs[k] + xs[k + 1]) + (ys[k] + ys[k + g.pitch]);
    local = isfinite(r) ? fmax(0.0, r) : kInf;
  }
  local = warp_max(local);
  if ((tid & 31) == 0) s_max[tid >> 5] = local;
  __syncthreads();
  if (tid == 0) {
    double m = s_max[0];
    for (int w = 1; w < 8; ++w) m = fmax(m, s_max[w]);
    atomicMax(&ctl->max_rate, dbits(m));
  }
}

template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_cell_emf_s(Grid g, StateP u, double* cell_ez,
                                                    const double* xs, const double* ys,
                                                    int cfl_reduce, double gamma, Ctl* ctl) {
  b_cell_emf_s<ORDER>(g, u, cell_ez, xs, ys, cfl_reduce, gamma, ctl, blockIdx.x, blockIdx.y);
}

// The same with the tile staged by TMA from the register's tensor map
// (single-instance path; this GPU's own memory, no multicast).
template <int ORDER>
__global__ void __launch_bounds__(256, 3) k_cell_emf_tma(Grid g, StateP u,
                                                      const __grid_constant__ CUtensorMap map,
                                                      double* cell_ez, const double* xs,
                                                      const double* ys, int cfl_reduce,
                                                      double gamma, Ctl* ctl) {
  b_cell_emf_s<ORDER, true>(g, u, cell_ez, xs, ys, cfl_reduce, gamma, ctl, blockIdx.x,
                            blockIdx.y, &map);
}

// Face -> edge interpolation (mhd_ct.hip:50-97) with the constant shortcut.
template <int NT>
__device__ __forceinline__ double edge_interp(const double* e) {
  bool same = true;
#pragma unroll
  for (int q = 1; q < NT; ++q) same = same && (e[q] == e[0]);
  if (same) return e[0];
  if (NT == 2) return __dmul_rn(__dadd_rn(e[0], e[1]), 0.5);  // = / 2 exactly
  if (NT == 6)
    return (((((e[0] - 8.0 * e[1]) + 37.0 * e[2]) + 37.0 * e[3]) - 8.0 * e[4]) + e[5]) / 60.0;
  return (((((((-3.0 * e[0] + 29.0 * e[1]) - 139.0 * e[2]) + 533.0 * e[3]) + 533.0 * e[4]) -
            139.0 * e[5]) + 29.0 * e[6]) - 3.0 * e[7]) / 840.0;
}

// Upwind CT corner E_z = ex + ey - centred, with the exact one-dimensional
// limits (mhd_ct.hip:811-878).
template <int ORDER>
__global__ void __launch_bounds__(128) k_corner_emf(Grid g, const double* cell_ez,
                                                    const double* xemf, const double* yemf,
                                                    const int* xnj, const int* ynj, double* ez,
                                                    const Ctl* ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.nx || j > g.ny) return;
  if (ctl->status) return;
  const long long k = g.idx(i, j);
  const bool conducting = (i == 0 && g.bc[0] == 2) || (i == g.nx && g.bc[1] == 2) ||
                          (j == 0 && g.bc[2] == 2) || (j == g.ny && g.bc[3] == 2);
  if (conducting) {
    ez[k] = 0.0;
    return;
  }
  constexpr int LO = ORDER >= 7 ? -4 : ORDER >= 5 ? -3 : -1;
  constexpr int NT = ORDER >= 7 ? 8 : ORDER >= 5 ? 6 : 2;
  int mi[NT], mj[NT];
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    mi[q] = face_index(i + LO + q, g.nx, g.bc[0], g.bc[1]);
    mj[q] = face_index(j + LO + q, g.ny, g.bc[2], g.bc[3]);
  }
  const int fi = face_index(i, g.nx, g.bc[0], g.bc[1]);
  const int fj = face_index(j, g.ny, g.bc[2], g.bc[3]);
  double e[NT], line[NT];
#pragma unroll
  for (int q = 0; q < NT; ++q) e[q] = xemf[g.idx(fi, mj[q])];
  const double ex = edge_interp<NT>(e);
#pragma unroll
  for (int q = 0; q < NT; ++q) e[q] = yemf[g.idx(mi[q], fj)];
  const double ey = edge_interp<NT>(e);
  // cell-centred reference, and the constancy of the cell table along x
  // (y_only) and along y (x_only) over the same stencil
  bool const_x = true, const_y = true;
  double col0[NT];
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    double c[NT];
#pragma unroll
    for (int p = 0; p < NT; ++p) c[p] = cell_ez[g.idx(mi[p], mj[q])];
#pragma unroll
    for (int p = 1; p < NT; ++p) const_x = const_x && (c[p] == c[0]);
    if (q == 0) {
#pragma unroll
      for (int p = 0; p < NT; ++p) col0[p] = c[p];
    } else {
#pragma unroll
      for (int p = 0; p < NT; ++p) const_y = const_y && (c[p] == col0[p]);
    }
    line[q] = edge_interp<NT>(c);
  }
  const double centred = edge_interp<NT>(line);
  bool nj_y = true, nj_x = true;
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    const int a = mi[q], b = mj[q];
    nj_y = nj_y && in_pad(g, a, fj) && ynj[g.idx(a, fj)] != 0;
    nj_x = nj_x && in_pad(g, fi, b) && xnj[g.idx(fi, b)] != 0;
  }
  const bool x_only = nj_y && const_y;
  const bool y_only = nj_x && const_x;
  double v;
  if (x_only && !y_only) v = ex;
  else if (y_only && !x_only) v = ey;
  else v = crsum3(ex, ey, -centred);
  ez[k] = v;
}

// Same corner EMF with the block's cell E_z stencil staged in shared memory:
// a (32 + NT - 1) x (4 + NT - 1) tile of the mapped cell table, so each
// corner's NT x NT reads are shared-memory loads.  Tile coordinates go
// through face_index like every CT table read, which keeps them inside the
// padded grid for any block position.
template <int ORDER>
__device__ __forceinline__ void b_corner_emf_s(const Grid& g, const double* cell_ez, const double* xemf,
                                               const double* yemf, const int* xnj, const int* ynj,
                                               double* ez, const Ctl* ctl, int bx, int by) {
  constexpr int LO = ORDER >= 7 ? -4 : ORDER >= 5 ? -3 : -1;
  constexpr int NT = ORDER >= 7 ? 8 : ORDER >= 5 ? 6 : 2;
  constexpr int TW = 32 + NT - 1, TH = 4 + NT - 1;
  // the block's mapped stencils: cell E_z (TH x TW), the x-face E_z and proofs
  // of its 32 corner columns over TH rows, the y-face ones of its 4 corner
  // rows over TW columns
  __shared__ double tile[TH][TW];
  __shared__ double sxe[TH][32], sye[4][TW];
  __shared__ int sxn[TH][32], syn[4][TW];
  // separable centred value: each tile row's x-interpolation at the block's
  // 32 corner columns (xr), whether that row is constant over the corner's
  // x-stencil (xc), and whether each tile column is constant over the y-
  // stencil of each of the 4 corner rows (yc); every corner then reads NT of
  // each instead of its NT x NT cells (same sums, same order)
  __shared__ double xr[TH][32];
  __shared__ unsigned char xc[TH][32], yc[4][TW];
  if (ctl->status) return;  // uniform over the block
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
  const int i0 = bx * 32, j0 = by * 4;
  for (int t = tid; t < TH * TW; t += 128) {
    const int a = t % TW, b = t / TW;
    const int mi = face_index(i0 + LO + a, g.nx, g.bc[0], g.bc[1]);
    const int mj = face_index(j0 + LO + b, g.ny, g.bc[2], g.bc[3]);
    tile[b][a] = __ldg(cell_ez + g.idx(mi, mj));
  }
  for (int t = tid; t < TH * 32; t += 128) {
    const int a = t % 32, b = t / 32;
    const int fi = face_index(i0 + a, g.nx, g.bc[0], g.bc[1]);
    const int mj = face_index(j0 + LO + b, g.ny, g.bc[2], g.bc[3]);
    const long long kx = g.idx(fi, mj);
    sxe[b][a] = __ldg(xemf + kx);
    sxn[b][a] = __ldg(xnj + kx);
  }
  for (int t = tid; t < 4 * TW; t += 128) {
    const int a = t % TW, b = t / TW;
    const int mi = face_index(i0 + LO + a, g.nx, g.bc[0], g.bc[1]);
    const int fj = face_index(j0 + b, g.ny, g.bc[2], g.bc[3]);
    const long long ky = g.idx(mi, fj);
    sye[b][a] = __ldg(yemf + ky);
    syn[b][a] = __ldg(ynj + ky);
  }
  __syncthreads();
  for (int t = tid; t < TH * 32; t += 128) {
    const int a = t % 32, b = t / 32;
    double c[NT];
#pragma unroll
    for (int p = 0; p < NT; ++p) c[p] = tile[b][a + p];
    bool cst = true;
#pragma unroll
    for (int p = 1; p < NT; ++p) cst = cst && (c[p] == c[0]);
    xr[b][a] = edge_interp<NT>(c);
    xc[b][a] = cst;
  }
  for (int t = tid; t < 4 * TW; t += 128) {
    const int a = t % TW, b = t / TW;
    const double c0 = tile[b][a];
    bool cst = true;
#pragma unroll
    for (int q = 1; q < NT; ++q) cst = cst && (tile[b + q][a] == c0);
    yc[b][a] = cst;
  }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  if (i > g.nx || j > g.ny) return;
  const long long k = g.idx(i, j);
  const bool conducting = (i == 0 && g.bc[0] == 2) || (i == g.nx && g.bc[1] == 2) ||
                          (j == 0 && g.bc[2] == 2) || (j == g.ny && g.bc[3] == 2);
  if (conducting) {
    ez[k] = 0.0;
    return;
  }
  double e[NT], line[NT];
  bool nj_y = true, nj_x = true;
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    e[q] = sxe[ty + q][tx];
    nj_x = nj_x && sxn[ty + q][tx] != 0;
  }
  const double ex = edge_interp<NT>(e);
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    e[q] = sye[ty][tx + q];
    nj_y = nj_y && syn[ty][tx + q] != 0;
  }
  const double ey = edge_interp<NT>(e);
  bool const_x = true, const_y = true;
#pragma unroll
  for (int q = 0; q < NT; ++q) {
    line[q] = xr[ty + q][tx];
    const_x = const_x && xc[ty + q][tx];
    const_y = const_y && yc[ty][tx + q];
  }
  const double centred = edge_interp<NT>(line);
  const bool x_only = nj_y && const_y;
  const bool y_only = nj_x && const_x;
  double v;
  if (x_only && !y_only) v = ex;
  else if (y_only && !x_only) v = ey;
  else v = crsum3(ex, ey, -centred);
  ez[k] = v;
}

template <int ORDER>
__global__ void __launch_bounds__(128, 4) k_corner_emf_s(Grid g, const double* cell_ez,
                                                      const double* xemf, const double* yemf,
                                                      const int* xnj, const int* ynj, double* ez,
                                                      const Ctl* ctl) {
  b_corner_emf_s<ORDER>(g, cell_ez, xemf, yemf, xnj, ynj, ez, ctl, blockIdx.x, blockIdx.y);
}

// Flux difference + EMF curl + Shu-Osher combine (mhd_update.hip:21-206,
// mhd_ct.hip:893-931, mhd_solver.cpp:840-874).  Writes cells and the owned
// high faces of the output; ghosts are closed by fill_ghosts afterwards.
__device__ __forceinline__ void b_update(const Grid& g, const StateP& un, const StateP& us,
                                         const StateP& out, const FluxP& fx, const FluxP& fy,
                                         const double* ez, const double* dt_dev, double dt_host,
                                         int stage, const Ctl* ctl, int bx, int by) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  if (i > g.nx || j > g.ny) return;
  if (ctl->status) return;
  const double dt = dt_dev ? *dt_dev : dt_host;
  double a, b, c;
  if (stage == 0) {
    a = 1.0; b = 0.0; c = dt;
  } else if (stage == 1) {
    a = 3.0 / 4.0; b = 1.0 / 4.0; c = (1.0 / 4.0) * dt;
  } else {
    a = 1.0 / 3.0; b = 2.0 / 3.0; c = (2.0 / 3.0) * dt;
  }
  auto combine = [&](double vn, double vs, double d) {
    // rk_weighted_sum (mhd_update.hip:113-135): zero weights skip operands
    if (b == 0.0) return __dadd_rn(__dmul_rn(a, vn), __dmul_rn(c, d));
    return crsum3(__dmul_rn(a, vn), __dmul_rn(b, vs), __dmul_rn(c, d));
  };
  const long long k = g.idx(i, j);
  const double rdx = pow2_recip(g.dx), rdy = pow2_recip(g.dy);
  if (i < g.nx && j < g.ny) {
    const int cc[6] = {0, 1, 2, 3, 4, 7};
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const int q = cc[t];
      const double dqx =
          __dadd_rn(div_by(fx.f[q][k + 1], g.dx, rdx), div_by(-fx.f[q][k], g.dx, rdx));
      const double dqy =
          __dadd_rn(div_by(fy.f[q][k + g.pitch], g.dy, rdy), div_by(-fy.f[q][k], g.dy, rdy));
      const double d = __dadd_rn(-dqx, -dqy);
      out.c[q][k] = combine(un.c[q][k], b == 0.0 ? 0.0 : us.c[q][k], d);
    }
  }
  if (j < g.ny) {
    const double d = __dadd_rn(div_by(-ez[k + g.pitch], g.dy, rdy), div_by(ez[k], g.dy, rdy));
    out.c[5][k] = combine(un.c[5][k], b == 0.0 ? 0.0 : us.c[5][k], d);
  }
  if (i < g.nx) {
    const double d = __dadd_rn(div_by(ez[k + 1], g.dx, rdx), div_by(-ez[k], g.dx, rdx));
    out.c[6][k] = combine(un.c[6][k], b == 0.0 ? 0.0 : us.c[6][k], d);
  }
}

// b_update two cells at a time, every load and store of the pair one
// 16-byte double2 access (the pair's first padded column is even and the
// pitch is even, so each pair is aligned); the per-cell arithmetic and the
// cells written are b_update's.  Reads of the pair's partner beyond the
// updated range stay inside the padded arrays (ng >= 3).
__device__ __forceinline__ double2 ld2(const double* p) {
  return __ldg(reinterpret_cast<const double2*>(p));
}
__device__ __forceinline__ void st_pair(double* p, bool a, bool b, double va, double vb) {
  if (a && b) *reinterpret_cast<double2*>(p) = make_double2(va, vb);
  else if (a) p[0] = va;
  else if (b) p[1] = vb;
}
__global__ void __launch_bounds__(256) k_update2(Grid g, StateP un, StateP us, StateP out,
                                                 FluxP fx, FluxP fy, const double* ez,
                                                 const double* dt_dev, double dt_host, int stage,
                                                 const Ctl* ctl) {
  const int pr = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int ia = 2 * pr - g.ng;  // the pair is cells ia, ia + 1 (padded columns 2 pr, 2 pr + 1)
  if (ia > g.nx || j > g.ny) return;
  if (ctl->status) return;
  const double dt = dt_dev ? *dt_dev : dt_host;
  double a, b, c;
  if (stage == 0) {
    a = 1.0; b = 0.0; c = dt;
  } else if (stage == 1) {
    a = 3.0 / 4.0; b = 1.0 / 4.0; c = (1.0 / 4.0) * dt;
  } else {
    a = 1.0 / 3.0; b = 2.0 / 3.0; c = (2.0 / 3.0) * dt;
  }
  auto combine = [&](double vn, double vs, double d) {
    if (b == 0.0) return __dadd_rn(__dmul_rn(a, vn), __dmul_rn(c, d));
    return crsum3(__dmul_rn(a, vn), __dmul_rn(b, vs), __dmul_rn(c, d));
  };
  const long long k = g.idx(ia, j), P = g.pitch;
  const double rdx = pow2_recip(g.dx), rdy = pow2_recip(g.dy);
  const int ib = ia + 1;
  // cell-centred components: i < nx, j < ny
  const bool ca = j < g.ny && ia >= 0 && ia < g.nx, cb = j < g.ny && ib >= 0 && ib < g.nx;
  if (ca || cb) {
    const int cc[6] = {0, 1, 2, 3, 4, 7};
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const int q = cc[t];
      const double2 x01 = ld2(fx.f[q] + k);
      const double x2 = __ldg(fx.f[q] + k + 2);
      const double2 y0 = ld2(fy.f[q] + k), y1 = ld2(fy.f[q] + k + P);
      const double dxa = __dadd_rn(div_by(x01.y, g.dx, rdx), div_by(-x01.x, g.dx, rdx));
      const double dxb = __dadd_rn(div_by(x2, g.dx, rdx), div_by(-x01.y, g.dx, rdx));
      const double dya = __dadd_rn(div_by(y1.x, g.dy, rdy), div_by(-y0.x, g.dy, rdy));
      const double dyb = __dadd_rn(div_by(y1.y, g.dy, rdy), div_by(-y0.y, g.dy, rdy));
      const double2 vn = ld2(un.c[q] + k);
      const double2 vs = b == 0.0 ? make_double2(0.0, 0.0) : ld2(us.c[q] + k);
      st_pair(out.c[q] + k, ca, cb, combine(vn.x, vs.x, __dadd_rn(-dxa, -dya)),
              combine(vn.y, vs.y, __dadd_rn(-dxb, -dyb)));
    }
  }
  const double2 e0 = ld2(ez + k);
  // x-face field: i <= nx, j < ny
  const bool fa = j < g.ny && ia >= 0, fb = j < g.ny && ib >= 0 && ib <= g.nx;
  if (fa || fb) {
    const double2 e1 = ld2(ez + k + P);
    const double2 vn = ld2(un.c[5] + k);
    const double2 vs = b == 0.0 ? make_double2(0.0, 0.0) : ld2(us.c[5] + k);
    const double da = __dadd_rn(div_by(-e1.x, g.dy, rdy), div_by(e0.x, g.dy, rdy));
    const double db = __dadd_rn(div_by(-e1.y, g.dy, rdy), div_by(e0.y, g.dy, rdy));
    st_pair(out.c[5] + k, fa, fb, combine(vn.x, vs.x, da), combine(vn.y, vs.y, db));
  }
  // y-face field: i < nx, j <= ny
  const bool ha = ia >= 0 && ia < g.nx, hb = ib >= 0 && ib < g.nx;
  if (ha || hb) {
    const double e2 = __ldg(ez + k + 2);
    const double2 vn = ld2(un.c[6] + k);
    const double2 vs = b == 0.0 ? make_double2(0.0, 0.0) : ld2(us.c[6] + k);
    const double da = __dadd_rn(div_by(e0.y, g.dx, rdx), div_by(-e0.x, g.dx, rdx));
    const double db = __dadd_rn(div_by(e2, g.dx, rdx), div_by(-e0.y, g.dx, rdx));
    st_pair(out.c[6] + k, ha, hb, combine(vn.x, vs.x, da), combine(vn.y, vs.y, db));
  }
}

__global__ void __launch_bounds__(256) k_update(Grid g, StateP un, StateP us, StateP out,
                                                FluxP fx, FluxP fy, const double* ez,
                                                const double* dt_dev, double dt_host, int stage,
                                                const Ctl* ctl) {
  b_update(g, un, us, out, fx, fy, ez, dt_dev, dt_host, stage, ctl, blockIdx.x, blockIdx.y);
}

// Consume the live-state preflights computed with the previous state and
// reset the per-step reductions.  coll selects which collocation the
// admissibility preflight uses (mhd_solver.cpp:689-692); anchor_mode >= 0
// forces the low-order anchor flag, -1 derives it from the live state.
__device__ __forceinline__ void k_step_begin_body(Ctl* ctl, int coll, int anchor_mode) {
  if (ctl->status) return;
  int st = 0;
  if ((coll ? ctl->anchor_theta : ctl->live_theta) != dbits(1.0)) st |= kStatusNotAdmissible;
  const double res = __longlong_as_double((long long)ctl->divb_res);
  const double sc = __longlong_as_double((long long)ctl->divb_scale);
  const double rel = res == 0.0 ? 0.0 : res / sc;
  if (!(isfinite(rel) && rel <= 1024.0 * kEps)) st |= kStatusNotSolenoidal;
  ctl->anchor_ok = anchor_mode >= 0 ? anchor_mode : (ctl->anchor_theta == dbits(1.0) ? 1 : 0);
  ctl->status = st;
  ctl->theta = dbits(1.0);
  ctl->max_rate = 0ull;
  ctl->live_theta = dbits(1.0);
  ctl->anchor_theta = dbits(1.0);
  ctl->divb_res = 0ull;
  ctl->divb_scale = 0ull;
}
__global__ void k_step_begin(Ctl* ctl, int coll, int anchor_mode) { k_step_begin_body(ctl, coll, anchor_mode); }

// Clear the status word and the live-state accumulators before the live
// state's preflights are recomputed.
__global__ void k_reset_stats(Ctl* ctl) {
  ctl->status = 0;
  ctl->live_theta = dbits(1.0);
  ctl->anchor_theta = dbits(1.0);
  ctl->divb_res = 0ull;
  ctl->divb_scale = 0ull;
}

__device__ __forceinline__ void k_set_time_body(Ctl* ctl, double t, double t_end) {
  ctl->t = t;
  ctl->t_end = t_end;
  ctl->steps_done = 0;
  ctl->status = 0;
}
__global__ void k_set_time(Ctl* ctl, double t, double t_end) { k_set_time_body(ctl, t, t_end); }

// dt = cfl_eff / max_rate (mhd_solver.cpp:1283-1320), optionally clipped to
// the remaining interval of a device-resident run.
__device__ __forceinline__ void k_dt_body(Ctl* ctl, double cfl_eff, double hmin, double hmax, int clip) {
  if (ctl->status) return;
  const double mr = __longlong_as_double((long long)ctl->max_rate);
  if (!isfinite(mr)) {
    ctl->status |= kStatusCflNonFinite;
    return;
  }
  double dt = mr > 0.0 ? cfl_eff / mr : cfl_eff * (hmin / (1.0 + hmin / hmax));
  if (clip) {
    const double rem = ctl->t_end - ctl->t;
    if (!(rem > 0.0)) {
      ctl->status |= kStatusDone;
      return;
    }
    dt = fmin(dt, rem);
  }
  ctl->dt = dt;
}
__global__ void k_dt(Ctl* ctl, double cfl_eff, double hmin, double hmax, int clip) { k_dt_body(ctl, cfl_eff, hmin, hmax, clip); }

__device__ __forceinline__ void k_step_end_body(Ctl* ctl) {
  if (ctl->status) return;
  const double rem = ctl->t_end - ctl->t;
  ctl->t = ctl->dt == rem ? ctl->t_end : ctl->t + ctl->dt;
  ctl->steps_done += 1;
  if (!(ctl->t < ctl->t_end)) ctl->status |= kStatusDone;
}
__global__ void k_step_end(Ctl* ctl) { k_step_end_body(ctl); }

__global__ void k_divb_linf(Grid g, StateP u, unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny || !g.in_window(i, j)) return;
  const long long k = g.idx(i, j);
  // ct_divb_linf_kernel (mhd_reduce.hip:505-553)
  const double rdx = pow2_recip(g.dx), rdy = pow2_recip(g.dy);
  const double d = __dadd_rn(__dadd_rn(div_by(u.c[5][k + 1], g.dx, rdx), div_by(-u.c[5][k], g.dx, rdx)),
                             __dadd_rn(div_by(u.c[6][k + g.pitch], g.dy, rdy),
                                       div_by(-u.c[6][k], g.dy, rdy)));
  const double v = isfinite(d) ? fabs(d) : kInf;
  atomic_max_lanes(out, v > 0.0 ? dbits(v) : 0ull);
}

// Per-block compensated partial sums of rho and energy over the cells.
__global__ void k_cell_sums(Grid g, StateP u, double* partial) {
  __shared__ double sm[2][256], sc[2][256];
  const int tid = threadIdx.x;
  double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
  const long long n = (long long)g.nx * g.ny;
  for (long long t = blockIdx.x * (long long)blockDim.x + tid; t < n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = int(t % g.nx), j = int(t / g.nx);
    if (!g.in_window(i, j)) continue;
    const long long k = g.idx(i, j);
    double e;
    two_sum(s0, u.c[0][k], s0, e);
    c0 += e;
    two_sum(s1, u.c[4][k], s1, e);
    c1 += e;
  }
  sm[0][tid] = s0; sc[0][tid] = c0;
  sm[1][tid] = s1; sc[1][tid] = c1;
  __syncthreads();
  if (tid == 0) {
    double a[2] = {0, 0}, ca[2] = {0, 0};
    for (int q = 0; q < 2; ++q)
      for (int t = 0; t < (int)blockDim.x; ++t) {
        double e;
        two_sum(a[q], sm[q][t], a[q], e);
        ca[q] += e + sc[q][t];
      }
    partial[4 * blockIdx.x + 0] = a[0];
    partial[4 * blockIdx.x + 1] = ca[0];
    partial[4 * blockIdx.x + 2] = a[1];
    partial[4 * blockIdx.x + 3] = ca[1];
  }
}

}  // namespace

// ===========================================================================
// Batched persistent kernels: each CTA walks the phase's tile list over all
// instances (stride gridDim.x), decodes (instance, tile) from the prefix
// table and runs the same device body as the single-instance kernel.
// ===========================================================================
namespace {

// (the component-wise pass, MODE 2, is memory-latency bound: 64 registers,
// eight blocks per SM; the characteristic pass needs 128)
template <int DIR, int ORDER, int MODE = 0>
__global__ void __launch_bounds__(128, MODE == 2 ? 8 : 4) kb_reconstruct(const BatchRec* __restrict__ r, BatchPlan p,
                                                      const BatchLearnRec* __restrict__ l = nullptr) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const int inst = batch_locate(p, t, &local);
    const BatchRec& q = r[inst];
    batch_block(DIR == 0 ? kBpRecon0 : kBpRecon1, q.a.g, local, &bx, &by);
    FaceList defer{};
    if (MODE == 2)
      defer = FaceList{l[inst].flag, DIR == 0 ? l[inst].xlist : l[inst].ylist,
                       l[inst].counts + DIR};
    b_reconstruct<DIR, ORDER, MODE>(q.a.g, q.a.u, DIR == 0 ? q.a.ix : q.a.iy, q.a.gamma,
                                    q.a.ctl, bx, by, nullptr, defer);
  }
}

// Characteristic pass over every instance's face list: each CTA takes its
// share of each instance's list in turn.
template <int DIR, int ORDER>
__global__ void __launch_bounds__(128, 4) kb_reconstruct_list(const BatchRec* __restrict__ r,
                                                              const BatchLearnRec* __restrict__ l,
                                                              int n) {
  // Work units are the 32-entry chunks of every instance's list, numbered
  // across the instances in order; warp w of the grid takes chunks w, w + W,
  // ... and walks the instances' chunk counts (device values, warp-uniform)
  // alongside, so that many small lists run side by side instead of one
  // list at a time.  A chunk is the same 32 entries the single-instance
  // list pass gives a warp.
  extern __shared__ double dsm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ws = dsm + warp * kWarpReconDoubles;
  const long long stride = (long long)gridDim.x * kReconWarps;
  long long c = (long long)blockIdx.x * kReconWarps + warp;  // this warp's next chunk
  long long first = 0;  // number of the first chunk of instance `inst`
  for (int inst = 0; inst < n;) {
    const BatchRec& q = r[inst];
    const int cnt = (q.a.ctl->status & ~kStatusDone) ? 0 : l[inst].counts[DIR];
    const long long chunks = (cnt + 31) / 32;
    if (c >= first + chunks) {
      first += chunks;
      ++inst;
      continue;
    }
    const int t = int(c - first) * 32 + lane;
    const bool valid = t < cnt;
    const Grid& g = q.a.g;
    int i = 0, j = 0;
    if (valid) {
      const int k = (DIR == 0 ? l[inst].xlist : l[inst].ylist)[t];
      i = k % g.pitch - g.ng;
      j = k / g.pitch - g.ng;
    }
    mp_faces_warp<DIR, ORDER>(g, q.a.u, DIR == 0 ? q.a.ix : q.a.iy, q.a.gamma, i, j, valid, ws);
    c += stride;
  }
}

__global__ void kb_learned_reset(const BatchRec* __restrict__ r, const BatchLearnRec* __restrict__ l,
                                 BatchPlan p) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local;
    const int inst = batch_locate(p, t, &local);
    const long long k = (long long)local * 256 + threadIdx.x;
    if (k < r[inst].a.g.size()) l[inst].flag[k] = 1;
    if (local == 0 && threadIdx.x < 2) l[inst].counts[threadIdx.x] = 0;
  }
}

// k_face_lists over 256-cell chunks of every instance.
__global__ void kb_face_lists(const BatchRec* __restrict__ r, const BatchLearnRec* __restrict__ l,
                              BatchPlan p) {
  for (int tt = blockIdx.x; tt < p.total; tt += gridDim.x) {
    int local;
    const int inst = batch_locate(p, tt, &local);
    const Grid& g = r[inst].a.g;
    const BatchLearnRec& L = l[inst];
    const long long t = (long long)local * 256 + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    bool nx_ = false, ny_ = false;
    const int k = int(t);
    if (t < g.size()) {
      const int i = int(t % g.pitch) - g.ng, j = int(t / g.pitch) - g.ng;
      if (i >= 0 && i <= g.nx && j < g.ny + g.ng) nx_ = (L.flag[t] | L.flag[t - 1]) != 0;
      if (j >= 0 && j <= g.ny && i < g.nx + g.ng) ny_ = (L.flag[t] | L.flag[t - g.pitch]) != 0;
    }
    const unsigned bx_ = __ballot_sync(0xffffffffu, nx_), by_ = __ballot_sync(0xffffffffu, ny_);
    int basex = 0, basey = 0;
    if (lane == 0) {
      if (bx_) basex = atomicAdd(&L.counts[0], __popc(bx_));
      if (by_) basey = atomicAdd(&L.counts[1], __popc(by_));
    }
    basex = __shfl_sync(0xffffffffu, basex, 0);
    basey = __shfl_sync(0xffffffffu, basey, 0);
    const unsigned below = (1u << lane) - 1u;
    if (nx_) L.xlist[basex + __popc(bx_ & below)] = k;
    if (ny_) L.ylist[basey + __popc(by_ & below)] = k;
  }
}

template <int DIR, int ORDER>
__global__ void __launch_bounds__(kFqThreads, kFqBlocksPerSm)
    kb_face_flux_q(const BatchRec* __restrict__ r, BatchPlan p, int speeds) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    batch_block(kBpFlux, q.a.g, local, &bx, &by);
    b_face_flux_qs<DIR, ORDER, kFqTX>(q.a.g, DIR == 0 ? q.a.ix : q.a.iy, DIR == 0 ? q.a.fx : q.a.fy,
                               DIR == 0 ? q.a.xemf : q.a.yemf, DIR == 0 ? q.a.xnj : q.a.ynj,
                               speeds ? (DIR == 0 ? q.a.xspd : q.a.yspd) : nullptr, q.a.gamma,
                               q.a.ctl, bx, by);
    __syncthreads();  // the shared tile is reused by the next tile
  }
}

template <int ORDER>
__global__ void __launch_bounds__(256, 3) kb_cell_emf_s(const BatchRec* __restrict__ r, BatchPlan p,
                                                     int cfl_reduce) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    batch_block(kBpCell, q.a.g, local, &bx, &by);
    b_cell_emf_s<ORDER>(q.a.g, q.a.u, q.a.cell_ez, q.a.xspd, q.a.yspd, cfl_reduce, q.a.gamma,
                        q.a.ctl, bx, by);
    __syncthreads();  // shared tiles are reused by the next tile
  }
}

template <int ORDER>
__global__ void __launch_bounds__(128, 4) kb_corner_emf_s(const BatchRec* __restrict__ r,
                                                          BatchPlan p) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    batch_block(kBpCorner, q.a.g, local, &bx, &by);
    b_corner_emf_s<ORDER>(q.a.g, q.a.cell_ez, q.a.xemf, q.a.yemf, q.a.xnj, q.a.ynj, q.a.ez,
                          q.a.ctl, bx, by);
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) kb_update(const BatchRec* __restrict__ r, BatchPlan p,
                                                 int stage) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    batch_block(kBpUpdate, q.a.g, local, &bx, &by);
    b_update(q.a.g, q.live, q.a.u, q.out, q.a.fx, q.a.fy, q.a.ez, &q.a.ctl->dt, 0.0, stage,
             q.a.ctl, bx, by);
  }
}

__global__ void __launch_bounds__(256) kb_fill_ghosts(const BatchRec* __restrict__ r, BatchPlan p,
                                                      int axis) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    b_fill_ghosts(q.a.g, q.out, axis, local);
  }
}

template <int W>
__global__ void __launch_bounds__(256, 3) kb_colloc_check(const BatchRec* __restrict__ r,
                                                       BatchPlan p, int theta_mask,
                                                       int live_checks) {
  for (int t = blockIdx.x; t < p.total; t += gridDim.x) {
    int local, bx, by;
    const BatchRec& q = r[batch_locate(p, t, &local)];
    batch_block(kBpColloc, q.a.g, local, &bx, &by);
    b_colloc_check<W>(q.a.g, q.out, q.live, 1, theta_mask, live_checks, 1, q.a.gamma, q.a.ctl,
                      bx, by);
  }
}

__global__ void kb_ctl(const BatchRec* __restrict__ r, int n, int what, double t0, double t_end) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const BatchRec& q = r[k];
  Ctl* ctl = q.a.ctl;
  if (what == 0) k_step_begin_body(ctl, 0, -1);
  else if (what == 1) k_dt_body(ctl, q.cfl_eff, q.hmin, q.hmax, 1);
  else if (what == 2) k_step_end_body(ctl);
  else k_set_time_body(ctl, t0, t_end);
}

}  // namespace

// ===========================================================================
// Launch wrappers
// ===========================================================================
namespace {
inline unsigned cdiv(long long a, int b) { return unsigned((a + b - 1) / b); }

// Raise a kernel's dynamic shared-memory limit once (per process).
void ensure_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::vector<const void*> done;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), fn) != done.end()) return;
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
  done.push_back(fn);
}
}  // namespace

void launch_fill_ghosts(const Grid& g, const StateP& u, cudaStream_t s) {
  for (int axis = 0; axis < 2; ++axis) {
    const long long n = 2LL * g.ng * ((axis == 0 ? g.ny : g.nx) + 2 * g.ng);
    k_fill_ghosts<<<cdiv(n, 256), 256, 0, s>>>(g, u, axis);
  }
}

void launch_colloc_check(const Grid& g, const StateP& cand, const StateP* base, int theta_mask,
                         bool /*anchor_check*/, bool live_checks, bool solver_owned,
                         double gamma, Ctl* ctl, cudaStream_t s) {
  const dim3 block(kBX, 8);
  const dim3 grid(cdiv(g.nx + 2 * g.ng, kBX), cdiv(g.ny + 2 * g.ng, 8));
  const StateP b = base ? *base : cand;
  const int hb = base ? 1 : 0;
  switch (g.ng) {
    case 2:
      k_colloc_check<4><<<grid, block, 0, s>>>(g, cand, b, hb, theta_mask, live_checks,
                                               solver_owned, gamma, ctl);
      break;
    case 3:
      k_colloc_check<6><<<grid, block, 0, s>>>(g, cand, b, hb, theta_mask, live_checks,
                                               solver_owned, gamma, ctl);
      break;
    default:
      k_colloc_check<8><<<grid, block, 0, s>>>(g, cand, b, hb, theta_mask, live_checks,
                                               solver_owned, gamma, ctl);
  }
}

template <int DIR, int ORDER>
static void recon_launch(const StageArgs& a, cudaStream_t s) {
  const Grid& g = a.g;

  const dim3 block(kBX, 4);
  const int ni = DIR == 0 ? g.nx + 1 : g.nx + 2 * g.ng;
  const int nj = DIR == 0 ? g.ny + 2 * g.ng : g.ny + 1;
  const dim3 grid(cdiv(ni, kBX), cdiv(nj, 4));
  size_t smem = 0;
  if (ORDER == 5 || ORDER == 7) {
    smem = kReconWarpSmem;
    ensure_smem((const void*)k_reconstruct<DIR, ORDER>, smem);
  }
  k_reconstruct<DIR, ORDER><<<grid, block, smem, s>>>(g, a.u, DIR == 0 ? a.ix : a.iy, a.gamma,
                                                      a.ctl);
}

void launch_reconstruct(const StageArgs& a, int dir, cudaStream_t s) {
#define QB_RECON(D, O) \
  if (dir == D && a.order == O) return recon_launch<D, O>(a, s);
  QB_RECON(0, 1) QB_RECON(1, 1) QB_RECON(0, 2) QB_RECON(1, 2)
  QB_RECON(0, 5) QB_RECON(1, 5) QB_RECON(0, 7) QB_RECON(1, 7)
#undef QB_RECON
}

template <int DIR, int ORDER>
static void flux_launch(const StageArgs& a, bool speeds, cudaStream_t s) {
  const Grid& g = a.g;
  if (ORDER == 5 || ORDER == 7) {
    constexpr int O = ORDER == 5 ? 5 : 7;
    const dim3 grid(cdiv(g.nx + 1, kFqTX), cdiv(g.ny + 1, fq_ty<O>()));
    k_face_flux_qs<DIR, O><<<grid, kFqThreads, 0, s>>>(
        g, DIR == 0 ? a.ix : a.iy, DIR == 0 ? a.fx : a.fy, DIR == 0 ? a.xemf : a.yemf,
        DIR == 0 ? a.xnj : a.ynj, speeds ? (DIR == 0 ? a.xspd : a.yspd) : nullptr, a.gamma, a.ctl);
    return;
  }
  const dim3 block(kBX, 4);
  const dim3 grid(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 4));
  k_face_flux<DIR, ORDER><<<grid, block, 0, s>>>(
      g, DIR == 0 ? a.ix : a.iy, DIR == 0 ? a.fx : a.fy, DIR == 0 ? a.xemf : a.yemf,
      DIR == 0 ? a.xnj : a.ynj, speeds ? (DIR == 0 ? a.xspd : a.yspd) : nullptr, a.gamma, a.ctl);
}

void launch_face_flux(const StageArgs& a, int dir, bool speeds, cudaStream_t s) {
#define QB_FLUX(D, O) \
  if (dir == D && a.order == O) return flux_launch<D, O>(a, speeds, s);
  QB_FLUX(0, 1) QB_FLUX(1, 1) QB_FLUX(0, 2) QB_FLUX(1, 2)
  QB_FLUX(0, 5) QB_FLUX(1, 5) QB_FLUX(0, 7) QB_FLUX(1, 7)
#undef QB_FLUX
}

template <int ORDER>
static void cell_tiled_launch(const StageArgs& a, bool cfl_reduce, cudaStream_t s) {
  const Grid& g = a.g;
  const dim3 grid(cdiv(g.nx + 1, kCellTX), cdiv(g.ny + 1, kCellTY));
  if (a.cell_map) {
    constexpr size_t tbytes = sizeof(double) * cell_smem_doubles<ORDER, true>();
    ensure_smem((const void*)k_cell_emf_tma<ORDER>, tbytes);
    k_cell_emf_tma<ORDER><<<grid, dim3(kCellTX, kCellTY), tbytes, s>>>(
        g, a.u, *a.cell_map, a.cell_ez, a.xspd, a.yspd, cfl_reduce ? 1 : 0, a.gamma, a.ctl);
    return;
  }
  constexpr size_t bytes = sizeof(double) * cell_smem_doubles<ORDER>();
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(k_cell_emf_s<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(bytes));
    configured = true;
  }
  k_cell_emf_s<ORDER><<<grid, dim3(kCellTX, kCellTY), bytes, s>>>(
      g, a.u, a.cell_ez, a.xspd, a.yspd, cfl_reduce ? 1 : 0, a.gamma, a.ctl);
}

void launch_cell_emf(const StageArgs& a, bool cfl_reduce, cudaStream_t s) {
  const Grid& g = a.g;
  if (a.order == 5) return cell_tiled_launch<5>(a, cfl_reduce, s);
  if (a.order == 7) return cell_tiled_launch<7>(a, cfl_reduce, s);
  const dim3 block(kBX, 4);
  const dim3 grid(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 4));
  const int r = cfl_reduce ? 1 : 0;
  switch (a.order) {
    case 1: k_cell_emf<1><<<grid, block, 0, s>>>(g, a.u, a.cell_ez, a.xspd, a.yspd, r, a.gamma, a.ctl); break;
    case 2: k_cell_emf<2><<<grid, block, 0, s>>>(g, a.u, a.cell_ez, a.xspd, a.yspd, r, a.gamma, a.ctl); break;
    case 5: k_cell_emf<5><<<grid, block, 0, s>>>(g, a.u, a.cell_ez, a.xspd, a.yspd, r, a.gamma, a.ctl); break;
    default: k_cell_emf<7><<<grid, block, 0, s>>>(g, a.u, a.cell_ez, a.xspd, a.yspd, r, a.gamma, a.ctl);
  }
}

bool make_state_tensor_map(const StateP& u, const Grid& g, int order, CUtensorMap* map) {
  if (order != 5 && order != 7) return false;
  const long long n = g.size();
  if ((g.pitch & 1) || (n & 1)) return false;  // 16-byte strides
  for (int c = 0; c < 8; ++c)
    if (u.c[c] != u.c[0] + c * n) return false;
  if (u.bxc != u.c[0] + 8 * n || u.byc != u.c[0] + 9 * n) return false;
  if (reinterpret_cast<uintptr_t>(u.c[0]) & 15) return false;
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  if (!encode) return false;
  const int sy = kCellTY + 2 * (order == 7 ? 3 : 2);
  cuuint64_t dims[3] = {cuuint64_t(g.pitch), cuuint64_t(g.ny + 2 * g.ng), 10};
  cuuint64_t strides[2] = {cuuint64_t(g.pitch) * sizeof(double), cuuint64_t(n) * sizeof(double)};
  cuuint32_t box[3] = {cuuint32_t(kTmaBW), cuuint32_t(sy), 1};
  cuuint32_t elem[3] = {1, 1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, u.c[0], dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

void launch_corner_emf(const StageArgs& a, cudaStream_t s) {
  const Grid& g = a.g;
  const dim3 block(kBX, 4);
  const dim3 grid(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 4));
  switch (a.order) {
    case 1:
    case 2: k_corner_emf<2><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl); break;
    case 5: k_corner_emf_s<5><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl); break;
    default: k_corner_emf_s<7><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl);
  }
}

void launch_update(const StageArgs& a, const StateP& un, const StateP& us, const StateP& out,
                   int stage, const double* dt_dev, double dt_host, cudaStream_t s) {
  const Grid& g = a.g;
  const dim3 block(kBX, 8);
  // the paired form needs an even pitch, at least three ghost layers and
  // 16-byte aligned arrays
  bool pairs = (g.pitch % 2) == 0 && g.ng >= 3;
  auto al = [](const double* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
  for (int q = 0; q < 8 && pairs; ++q)
    pairs = al(un.c[q]) && al(us.c[q]) && al(out.c[q]) && al(a.fx.f[q]) && al(a.fy.f[q]);
  pairs = pairs && al(a.ez);
  if (pairs) {
    const dim3 grid(cdiv((g.nx + g.ng + 2) / 2, kBX), cdiv(g.ny + 1, 8));
    k_update2<<<grid, block, 0, s>>>(g, un, us, out, a.fx, a.fy, a.ez, dt_dev, dt_host, stage,
                                     a.ctl);
    return;
  }
  const dim3 grid(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 8));
  k_update<<<grid, block, 0, s>>>(g, un, us, out, a.fx, a.fy, a.ez, dt_dev, dt_host, stage, a.ctl);
}

void launch_step_begin(Ctl* ctl, int coll, int anchor_mode, cudaStream_t s) {
  k_step_begin<<<1, 1, 0, s>>>(ctl, coll, anchor_mode);
}
void launch_reset_stats(Ctl* ctl, cudaStream_t s) { k_reset_stats<<<1, 1, 0, s>>>(ctl); }
void launch_set_time(Ctl* ctl, double t, double t_end, cudaStream_t s) {
  k_set_time<<<1, 1, 0, s>>>(ctl, t, t_end);
}

void launch_dt(Ctl* ctl, double cfl_eff, double hmin, double hmax, int clip, cudaStream_t s) {
  k_dt<<<1, 1, 0, s>>>(ctl, cfl_eff, hmin, hmax, clip);
}

void launch_step_end(Ctl* ctl, cudaStream_t s) { k_step_end<<<1, 1, 0, s>>>(ctl); }

void launch_divb_linf(const Grid& g, const StateP& u, unsigned long long* out, cudaStream_t s) {
  const dim3 block(kBX, 8);
  const dim3 grid(cdiv(g.nx, kBX), cdiv(g.ny, 8));
  k_divb_linf<<<grid, block, 0, s>>>(g, u, out);
}

void launch_cell_sums(const Grid& g, const StateP& u, double* partial, int blocks, cudaStream_t s) {
  k_cell_sums<<<blocks, 256, 0, s>>>(g, u, partial);
}

// ---- tile halo exchange on the device ---------------------------------------
// Gather and scatter one component by storage index.  Bad indices and
// non-finite values are recorded in *bad (bit 0: index outside [0, size),
// bit 1: non-finite value); the scatter runs as a check pass and a write
// pass, and the write pass does nothing once the check recorded a problem,
// so a rejected scatter leaves the component untouched.
__global__ void k_gather_values(const double* __restrict__ src, const long long* __restrict__ idx,
                                long long n, long long size, double* __restrict__ out,
                                unsigned long long* bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += stride) {
    const long long i = idx[k];
    if (i < 0 || i >= size) {
      atomicOr(bad, 1ull);
      out[k] = 0.0;
    } else {
      out[k] = src[i];
    }
  }
}

__global__ void k_scatter_check(const long long* __restrict__ idx, const double* __restrict__ v,
                                long long n, long long size, unsigned long long* bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  unsigned long long b = 0;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += stride) {
    const long long i = idx[k];
    if (i < 0 || i >= size) b |= 1ull;
    if (!isfinite(v[k])) b |= 2ull;
  }
  if (b) atomicOr(bad, b);
}

__global__ void k_scatter_values(double* __restrict__ dst, const long long* __restrict__ idx,
                                 const double* __restrict__ v, long long n,
                                 const unsigned long long* bad) {
  if (*bad) return;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += stride)
    dst[idx[k]] = v[k];
}

// Any non-finite value among v[0..n) sets *bad (which must start at zero).
__global__ void k_flag_nonfinite(const double* __restrict__ v, long long n,
                                 unsigned long long* bad) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  bool b = false;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += stride)
    b = b || !isfinite(v[k]);
  if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1ull);
}

namespace {
int exchange_blocks(long long n) {
  const long long b = (n + 255) / 256;
  return (int)(b < 4 * 148 ? (b > 0 ? b : 1) : 4 * 148);
}
}  // namespace

void launch_flag_nonfinite(const double* v, long long n, unsigned long long* bad, cudaStream_t s) {
  if (n <= 0) return;
  k_flag_nonfinite<<<exchange_blocks(n), 256, 0, s>>>(v, n, bad);
}

void launch_gather_values(const double* src, const long long* idx, long long n, long long size,
                          double* out, unsigned long long* bad, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_values<<<exchange_blocks(n), 256, 0, s>>>(src, idx, n, size, out, bad);
}

void launch_scatter_values(double* dst, const long long* idx, const double* v, long long n,
                           long long size, unsigned long long* bad, cudaStream_t s) {
  if (n <= 0) return;
  k_scatter_check<<<exchange_blocks(n), 256, 0, s>>>(idx, v, n, size, bad);
  k_scatter_values<<<exchange_blocks(n), 256, 0, s>>>(dst, idx, v, n, bad);
}

// ---- batched launchers -----------------------------------------------------
namespace {
template <class K>
int max_ctas(K kernel, int threads, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem) != cudaSuccess) b = 1;
  return b > 0 ? b : 1;
}
inline unsigned pgrid(const BatchPlan& p) { return unsigned(p.grid > 0 ? p.grid : p.total); }

template <int ORDER>
void batch_cell_configure() {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(kb_cell_emf_s<ORDER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(sizeof(double) * cell_smem_doubles<ORDER>()));
    done = true;
  }
}
}  // namespace

int batch_phase_threads(int phase) {
  switch (phase) {
    case kBpRecon0: case kBpRecon1: case kBpCorner: return 128;
    case kBpFlux: return kFqThreads;
    default: return 256;
  }
}

int batch_phase_max_ctas_per_sm(int phase, int order) {
  const bool o7 = order == 7;
  switch (phase) {
    case kBpRecon0:
      ensure_smem((const void*)kb_reconstruct<0, 7>, kReconWarpSmem);
      ensure_smem((const void*)kb_reconstruct<0, 5>, kReconWarpSmem);
      return o7 ? max_ctas(kb_reconstruct<0, 7>, 128, kReconWarpSmem)
                : max_ctas(kb_reconstruct<0, 5>, 128, kReconWarpSmem);
    case kBpRecon1:
      ensure_smem((const void*)kb_reconstruct<1, 7>, kReconWarpSmem);
      ensure_smem((const void*)kb_reconstruct<1, 5>, kReconWarpSmem);
      return o7 ? max_ctas(kb_reconstruct<1, 7>, 128, kReconWarpSmem)
                : max_ctas(kb_reconstruct<1, 5>, 128, kReconWarpSmem);
    case kBpFlux: {
      constexpr int t = kFqThreads;
      return o7 ? max_ctas(kb_face_flux_q<0, 7>, t, 0) : max_ctas(kb_face_flux_q<0, 5>, t, 0);
    }
    case kBpCell:
      if (o7) {
        batch_cell_configure<7>();
        return max_ctas(kb_cell_emf_s<7>, 256, sizeof(double) * cell_smem_doubles<7>());
      }
      batch_cell_configure<5>();
      return max_ctas(kb_cell_emf_s<5>, 256, sizeof(double) * cell_smem_doubles<5>());
    case kBpCorner: return o7 ? max_ctas(kb_corner_emf_s<7>, 128, 0) : max_ctas(kb_corner_emf_s<5>, 128, 0);
    case kBpUpdate: return max_ctas(kb_update, 256, 0);
    case kBpColloc: return o7 ? max_ctas(kb_colloc_check<8>, 256, 0) : max_ctas(kb_colloc_check<6>, 256, 0);
    default: return max_ctas(kb_fill_ghosts, 256, 0);
  }
}

void launch_batch_reconstruct(const BatchRec* r, const BatchPlan& p, int dir, int order,
                              cudaStream_t s) {
  const dim3 block(32, 4);
  if (order == 7) {
    if (dir == 0) {
      ensure_smem((const void*)kb_reconstruct<0, 7>, kReconWarpSmem);
      kb_reconstruct<0, 7><<<pgrid(p), block, kReconWarpSmem, s>>>(r, p);
    } else {
      ensure_smem((const void*)kb_reconstruct<1, 7>, kReconWarpSmem);
      kb_reconstruct<1, 7><<<pgrid(p), block, kReconWarpSmem, s>>>(r, p);
    }
  } else {
    if (dir == 0) {
      ensure_smem((const void*)kb_reconstruct<0, 5>, kReconWarpSmem);
      kb_reconstruct<0, 5><<<pgrid(p), block, kReconWarpSmem, s>>>(r, p);
    } else {
      ensure_smem((const void*)kb_reconstruct<1, 5>, kReconWarpSmem);
      kb_reconstruct<1, 5><<<pgrid(p), block, kReconWarpSmem, s>>>(r, p);
    }
  }
}

void launch_batch_face_flux(const BatchRec* r, const BatchPlan& p, int dir, int order,
                            bool speeds, cudaStream_t s) {
  const int sp = speeds ? 1 : 0;
  if (order == 7) {
    if (dir == 0) kb_face_flux_q<0, 7><<<pgrid(p), kFqThreads, 0, s>>>(r, p, sp);
    else kb_face_flux_q<1, 7><<<pgrid(p), kFqThreads, 0, s>>>(r, p, sp);
  } else {
    if (dir == 0) kb_face_flux_q<0, 5><<<pgrid(p), kFqThreads, 0, s>>>(r, p, sp);
    else kb_face_flux_q<1, 5><<<pgrid(p), kFqThreads, 0, s>>>(r, p, sp);
  }
}

void launch_batch_cell_emf(const BatchRec* r, const BatchPlan& p, int order, bool cfl_reduce,
                           cudaStream_t s) {
  const dim3 block(kCellTX, kCellTY);
  if (order == 7) {
    batch_cell_configure<7>();
    kb_cell_emf_s<7><<<pgrid(p), block, sizeof(double) * cell_smem_doubles<7>(), s>>>(
        r, p, cfl_reduce ? 1 : 0);
  } else {
    batch_cell_configure<5>();
    kb_cell_emf_s<5><<<pgrid(p), block, sizeof(double) * cell_smem_doubles<5>(), s>>>(
        r, p, cfl_reduce ? 1 : 0);
  }
}

void launch_batch_corner_emf(const BatchRec* r, const BatchPlan& p, int order, cudaStream_t s) {
  const dim3 block(32, 4);
  if (order == 7) kb_corner_emf_s<7><<<pgrid(p), block, 0, s>>>(r, p);
  else kb_corner_emf_s<5><<<pgrid(p), block, 0, s>>>(r, p);
}

void launch_batch_update(const BatchRec* r, const BatchPlan& p, int stage, cudaStream_t s) {
  kb_update<<<pgrid(p), dim3(32, 8), 0, s>>>(r, p, stage);
}

void launch_batch_fill_ghosts(const BatchRec* r, const BatchPlan& p, int axis, cudaStream_t s) {
  kb_fill_ghosts<<<pgrid(p), 256, 0, s>>>(r, p, axis);
}

void launch_batch_colloc_check(const BatchRec* r, const BatchPlan& p, int order, int theta_mask,
                               bool live_checks, cudaStream_t s) {
  const dim3 block(32, 8);
  if (order == 7) kb_colloc_check<8><<<pgrid(p), block, 0, s>>>(r, p, theta_mask, live_checks ? 1 : 0);
  else kb_colloc_check<6><<<pgrid(p), block, 0, s>>>(r, p, theta_mask, live_checks ? 1 : 0);
}

void launch_batch_learned_reset(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& cells,
                                cudaStream_t s) {
  kb_learned_reset<<<pgrid(cells), 256, 0, s>>>(r, l, cells);
}

void launch_batch_face_lists(const BatchRec* r, const BatchLearnRec* l, const BatchPlan& cells,
                             cudaStream_t s) {
  kb_face_lists<<<pgrid(cells), 256, 0, s>>>(r, l, cells);
}

void launch_batch_reconstruct_learned(const BatchRec* r, const BatchLearnRec* l,
                                      const BatchPlan& p, int dir, int order, int list_grid,
                                      cudaStream_t s) {
  const dim3 block(32, 4);
  if (order == 7) {
    if (dir == 0) {
      kb_reconstruct<0, 7, 2><<<pgrid(p), block, 0, s>>>(r, p, l);
      ensure_smem((const void*)kb_reconstruct_list<0, 7>, kReconWarpSmem);
      kb_reconstruct_list<0, 7><<<list_grid, 128, kReconWarpSmem, s>>>(r, l, p.n);
    } else {
      kb_reconstruct<1, 7, 2><<<pgrid(p), block, 0, s>>>(r, p, l);
      ensure_smem((const void*)kb_reconstruct_list<1, 7>, kReconWarpSmem);
      kb_reconstruct_list<1, 7><<<list_grid, 128, kReconWarpSmem, s>>>(r, l, p.n);
    }
  } else {
    if (dir == 0) {
      kb_reconstruct<0, 5, 2><<<pgrid(p), block, 0, s>>>(r, p, l);
      ensure_smem((const void*)kb_reconstruct_list<0, 5>, kReconWarpSmem);
      kb_reconstruct_list<0, 5><<<list_grid, 128, kReconWarpSmem, s>>>(r, l, p.n);
    } else {
      kb_reconstruct<1, 5, 2><<<pgrid(p), block, 0, s>>>(r, p, l);
      ensure_smem((const void*)kb_reconstruct_list<1, 5>, kReconWarpSmem);
      kb_reconstruct_list<1, 5><<<list_grid, 128, kReconWarpSmem, s>>>(r, l, p.n);
    }
  }
}

void launch_batch_ctl(const BatchRec* r, int n, int what, double t, double t_end, cudaStream_t s) {
  kb_ctl<<<cdiv(n, 128), 128, 0, s>>>(r, n, what, t, t_end);
}

// ---- learned-mode reconstruction and indicator training data ----------------
namespace {
template <int DIR, int ORDER>
dim3 recon_grid(const Grid& g) {
  const int ni = DIR == 0 ? g.nx + 1 : g.nx + 2 * g.ng;
  const int nj = DIR == 0 ? g.ny + 2 * g.ng : g.ny + 1;
  return dim3(cdiv(ni, kBX), cdiv(nj, 4));
}
}  // namespace

void launch_reconstruct_label(const StageArgs& a, int dir, int* label, int literal,
                              cudaStream_t s) {
  const dim3 block(kBX, 4);
  const IfaceP out = dir == 0 ? a.ix : a.iy;
#define QB_LBL(D, O)                                                                          \
  if (dir == D && a.order == O) {                                                            \
    ensure_smem((const void*)k_reconstruct_label<D, O>, kReconSmem);                          \
    return (void)k_reconstruct_label<D, O><<<recon_grid<D, O>(a.g), block, kReconSmem, s>>>( \
        a.g, a.u, out, a.gamma, a.ctl, label, literal);                                       \
  }
  QB_LBL(0, 5) QB_LBL(1, 5) QB_LBL(0, 7) QB_LBL(1, 7)
#undef QB_LBL
}

void launch_reconstruct_learned(const StageArgs& a, int dir, const unsigned char* flag, int* list,
                                int* count, int list_grid, cudaStream_t s) {
  const dim3 block(kBX, 4);
  const IfaceP out = dir == 0 ? a.ix : a.iy;
  const FaceList defer{flag, list, count};
#define QB_LRN(D, O)                                                                            \
  if (dir == D && a.order == O) {                                                              \
    k_reconstruct_lin<D, O><<<recon_grid<D, O>(a.g), block, 0, s>>>(a.g, a.u, out, a.gamma,    \
                                                                    a.ctl, defer);             \
    ensure_smem((const void*)k_reconstruct_list<D, O>, kReconWarpSmem);                         \
    k_reconstruct_list<D, O><<<list_grid, 128, kReconWarpSmem, s>>>(a.g, a.u, out, a.gamma, a.ctl,   \
                                                                list, count);                  \
    return;                                                                                    \
  }
  QB_LRN(0, 5) QB_LRN(1, 5) QB_LRN(0, 7) QB_LRN(1, 7)
#undef QB_LRN
}

void launch_face_lists(const Grid& g, const unsigned char* flag, int* xlist, int* ylist,
                       int* counts, cudaStream_t s) {
  cudaMemsetAsync(counts, 0, 2 * sizeof(int), s);
  k_face_lists<<<cdiv(g.size(), 256), 256, 0, s>>>(g, flag, xlist, ylist, counts);
}

// ===========================================================================
// Kernels of the per-kernel launch interface (reference
// include/quasar/physics/mhd/kernels.hpp): the pieces that the fused step
// above combines (flux difference, EMF curl, stage combine) as separate
// launches, plus standalone forms of the reductions and fills.  Each uses the
// arithmetic of the fused kernel it stands beside, so a step composed from
// these launches reproduces the fused step.
// ===========================================================================
namespace {

// Never written: the status word every stage kernel polls reads 0.
__device__ Ctl g_abi_zero_ctl;

// dudt += -(F_hi - F_lo)/h over the interior cells, all eight slots
// (mhd_update.hip:21-105).
__global__ void __launch_bounds__(256) k_abi_flux_difference(Grid g, FluxP f, int dir, FluxP d) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const long long k = g.idx(i, j), kp = k + (dir == 0 ? 1 : g.pitch);
  const double h = dir == 0 ? g.dx : g.dy, rh = pow2_recip(h);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double dq = __dadd_rn(div_by(f.f[q][kp], h, rh), div_by(-f.f[q][k], h, rh));
    d.f[q][k] = __dadd_rn(d.f[q][k], -dq);
  }
}

// dudt.bx_face / dudt.by_face = curl of the corner E_z, overwritten
// (mhd_ct.hip:893-931): bx on i <= nx, j < ny; by on i < nx, j <= ny.
__global__ void __launch_bounds__(256) k_abi_curl_rate(Grid g, const double* __restrict__ ez,
                                                       double* dbx, double* dby) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.nx || j > g.ny) return;
  const long long k = g.idx(i, j);
  const double rdx = pow2_recip(g.dx), rdy = pow2_recip(g.dy);
  if (j < g.ny) dbx[k] = __dadd_rn(div_by(-ez[k + g.pitch], g.dy, rdy), div_by(ez[k], g.dy, rdy));
  if (i < g.nx) dby[k] = __dadd_rn(div_by(ez[k + 1], g.dx, rdx), div_by(-ez[k], g.dx, rdx));
}

// out = a un + b us + c dudt (mhd_update.hip:113-206): an operand whose weight
// is zero is not read, (1, 0, 0) is an exact copy; cell components over the
// interior, bx also on i = nx and by on j = ny.
__global__ void __launch_bounds__(256) k_abi_rk_stage(Grid g, StateP out, StateP un, StateP us,
                                                      FluxP d, double a, double b, double c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i > g.nx || j > g.ny) return;
  const long long k = g.idx(i, j);
  const bool copy = a == 1.0 && b == 0.0 && c == 0.0;
  const bool ua = a != 0.0, ub = b != 0.0, uc = c != 0.0;
  auto comb = [&](int q) {
    if (copy) return un.c[q][k];
    if (ua && ub && uc)
      return crsum3(__dmul_rn(a, un.c[q][k]), __dmul_rn(b, us.c[q][k]), __dmul_rn(c, d.f[q][k]));
    if (ua && ub) return __dadd_rn(__dmul_rn(a, un.c[q][k]), __dmul_rn(b, us.c[q][k]));
    if (ua && uc) return __dadd_rn(__dmul_rn(a, un.c[q][k]), __dmul_rn(c, d.f[q][k]));
    if (ub && uc) return __dadd_rn(__dmul_rn(b, us.c[q][k]), __dmul_rn(c, d.f[q][k]));
    if (ua) return __dmul_rn(a, un.c[q][k]);
    if (ub) return __dmul_rn(b, us.c[q][k]);
    if (uc) return __dmul_rn(c, d.f[q][k]);
    return 0.0;
  };
  if (i < g.nx && j < g.ny) {
    const int cc[6] = {0, 1, 2, 3, 4, 7};
#pragma unroll
    for (int t = 0; t < 6; ++t) out.c[cc[t]][k] = comb(cc[t]);
  }
  if (j < g.ny) out.c[5][k] = comb(5);
  if (i < g.nx) out.c[6][k] = comb(6);
}

// Face -> cell collocation of one axis over the padded grid
// (launch_mhd_collocate_face_to_cell, mhd_staggering.hpp:77-236).
template <int W>
__global__ void k_abi_collocate(Grid g, int axis, const double* __restrict__ face,
                                double* __restrict__ cell) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - g.ng;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - g.ng;
  if (i >= g.nx + g.ng || j >= g.ny + g.ng) return;
  cell[g.idx(i, j)] = axis == 0
                          ? face_to_cell<W>(face, (long long)g.idx(0, j), 1, i, -g.ng, g.nx + g.ng - 1)
                          : face_to_cell<W>(face, (long long)g.idx(i, 0), g.pitch, j, -g.ng,
                                            g.ny + g.ng - 1);
}

// ---- analytic initial state (mhd_initial_conditions.hip:59-340) -----------
// Status bits of kernels.hpp:650-655.
constexpr int kSeedDensity = 1, kSeedPressure = 2, kSeedMomentum = 4, kSeedEnergy = 8,
              kSeedCollocation = 16, kSeedCoordinate = 32;

struct SeedW {
  double rho, p, vx, vy, vz, bx, by, bz, eoff;
};

// The generators in the reference's operation order, every product and sum
// rounded on its own (no contraction); sin, cos and hypot are CUDA's.
__device__ SeedW seed_eval(const SeedSpec& s, int nx, double xc, double yc) {
  constexpr double kPi = 3.141592653589793;  // nearest double to pi
  const double two_pi = 2.0 * kPi;
  SeedW w{};
  switch (s.kind) {
    case 0: {  // brio_wu: left/right primitive states split at x = interface
      const double* side = xc < s.interface_x ? s.left : s.right;
      w.rho = side[0]; w.p = side[1]; w.vx = side[2]; w.vy = side[3]; w.vz = side[4];
      w.bx = side[5]; w.by = side[6]; w.bz = side[7];
      break;
    }
    case 1: {  // alfven_wave along x with the sinc cell-average factor
      const double n = double(s.wavenumber);
      const double k = __ddiv_rn(__dmul_rn(two_pi, n), s.lx);
      const double phase = __dmul_rn(k, __dsub_rn(xc, s.ox));
      const double q = __ddiv_rn(n, double(nx));
      double fv = 1.0;
      if (q != 0.0) {
        const double pq = __dmul_rn(kPi, q);
        fv = __ddiv_rn(sin(pq), pq);
      }
      const double inv = __ddiv_rn(copysign(s.mvs, s.total_b0), __dsqrt_rn(s.rho));
      const double sp = sin(phase), cp = cos(phase);
      const double a = __dmul_rn(__dmul_rn(-s.amplitude, inv), fv);
      w.rho = s.rho; w.p = s.pressure; w.vx = 0.0;
      w.vy = __dmul_rn(a, sp);
      w.vz = __dmul_rn(a, cp);
      w.bx = s.b0;
      w.by = __dmul_rn(__dmul_rn(s.amplitude, fv), sp);
      w.bz = __dmul_rn(__dmul_rn(s.amplitude, fv), cp);
      const double sa = __dmul_rn(s.amplitude, s.mvs);
      w.eoff = __dmul_rn(__dmul_rn(sa, sa), __dsub_rn(1.0, __dmul_rn(fv, fv)));
      break;
    }
    case 2: {  // orszag_tang
      const double xi = __ddiv_rn(__dsub_rn(xc, s.ox), s.lx);
      const double eta = __ddiv_rn(__dsub_rn(yc, s.oy), s.ly);
      const double b0 = s.b_uniform[0];
      const double se = sin(__dmul_rn(two_pi, eta));
      w.rho = __dmul_rn(s.gamma, s.gamma); w.p = s.gamma;
      w.vx = -se;
      w.vy = sin(__dmul_rn(two_pi, xi));
      w.bx = __dmul_rn(-b0, se);
      w.by = __dmul_rn(b0, sin(__dmul_rn(2.0 * two_pi, xi)));
      break;
    }
    case 3: {  // blast: pressure disk
      const double r = hypot(__dsub_rn(xc, s.center[0]), __dsub_rn(yc, s.center[1]));
      w.rho = s.rho_ambient;
      w.p = r < s.r_in ? s.p_core : s.p_ambient;
      w.bx = s.b_uniform[0]; w.by = s.b_uniform[1]; w.bz = s.b_uniform[2];
      break;
    }
    case 4: {  // rotor: rigid disk with a linear taper
      const double rx = __dsub_rn(xc, s.center[0]), ry = __dsub_rn(yc, s.center[1]);
      const double r = hypot(rx, ry);
      double f = __ddiv_rn(__dsub_rn(s.r1, r), __dsub_rn(s.r1, s.r0));
      f = fmin(fmax(f, 0.0), 1.0);
      const bool inside = r <= s.r0;
      if (inside) f = 1.0;
      if (r >= s.r1) f = 0.0;
      double speed = 0.0;
      if (inside) speed = __ddiv_rn(s.u0, s.r0);
      else if (r < s.r1) speed = __ddiv_rn(__dmul_rn(f, s.u0), r);
      w.rho = __dadd_rn(s.rho_out, __dmul_rn(f, __dsub_rn(s.rho_in, s.rho_out)));
      w.p = s.p_ambient;
      w.vx = __dmul_rn(-speed, ry);
      w.vy = __dmul_rn(speed, rx);
      w.bx = s.b_uniform[0]; w.by = s.b_uniform[1]; w.bz = s.b_uniform[2];
      break;
    }
    default: {  // confined_blob: dense square, uniform bz
      const bool inside = fabs(__dsub_rn(xc, s.center[0])) <= s.blob_half &&
                          fabs(__dsub_rn(yc, s.center[1])) <= s.blob_half;
      w.rho = inside ? s.rho_in : s.rho_out;
      w.p = inside ? s.p_in : s.p_out;
      w.bz = s.b_uniform[2];
      break;
    }
  }
  return w;
}

// Pass 1 (mhd_initial_conditions.hip:211-282): one padded cell per thread;
// the faces of a cell take its centre value.
__global__ void __launch_bounds__(256) k_seed_pass1(Grid g, SeedSpec s, StateP u, double* raw,
                                                    int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - g.ng;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - g.ng;
  if (i >= g.nx + g.ng || j >= g.ny + g.ng) return;
  const double xc = fma(double(i) + 0.5, g.dx, s.ox);
  const double yc = fma(double(j) + 0.5, g.dy, s.oy);
  if (!(isfinite(xc) && isfinite(yc))) {
    atomicOr(status, kSeedCoordinate);
    return;
  }
  const SeedW w = seed_eval(s, g.nx, xc, yc);
  if (!(isfinite(w.rho) && w.rho > 0.0)) {
    atomicOr(status, kSeedDensity);
    return;
  }
  if (!(isfinite(w.p) && w.p > 0.0)) {
    atomicOr(status, kSeedPressure);
    return;
  }
  const double kinetic = kin_vel(w.rho, w.vx, w.vy, w.vz);
  const double magnetic = half_sq3(w.bx, w.by, w.bz);
  const double energy = __dadd_rn(
      __dadd_rn(__dadd_rn(__ddiv_rn(w.p, __dsub_rn(s.gamma, 1.0)), kinetic), magnetic), w.eoff);
  const double mx = __dmul_rn(w.rho, w.vx), my = __dmul_rn(w.rho, w.vy),
               mz = __dmul_rn(w.rho, w.vz);
  if (!(isfinite(mx) && isfinite(my) && isfinite(mz))) {
    atomicOr(status, kSeedMomentum);
    return;
  }
  if (!isfinite(energy)) {
    atomicOr(status, kSeedEnergy);
    return;
  }
  const long long k = g.idx(i, j);
  u.c[0][k] = w.rho;
  u.c[1][k] = mx;
  u.c[2][k] = my;
  u.c[3][k] = mz;
  u.c[4][k] = energy;
  u.c[5][k] = __dmul_rn(s.magnetic_scale, w.bx);
  u.c[6][k] = __dmul_rn(s.magnetic_scale, w.by);
  u.c[7][k] = __dmul_rn(s.magnetic_scale, w.bz);
  raw[k] = magnetic;
}

// Pass 2 (mhd_initial_conditions.hip:284-340): E = (E - raw) + |B_c|^2 / 2
// with B_c the collocated field the solver's EOS reads, then the preflight
// on the conserved arrays.
__global__ void __launch_bounds__(256) k_seed_recollocate(Grid g, double gamma, StateP u,
                                                          const double* raw, int* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - g.ng;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - g.ng;
  if (i >= g.nx + g.ng || j >= g.ny + g.ng) return;
  const long long k = g.idx(i, j);
  const double bxc = u.bxc[k], byc = u.byc[k];
  if (!(isfinite(bxc) && isfinite(byc))) {
    atomicOr(status, kSeedCollocation);
    return;
  }
  const double adjusted =
      __dadd_rn(__dsub_rn(u.c[4][k], raw[k]), half_sq3(bxc, byc, u.c[7][k]));
  if (!isfinite(adjusted)) {
    atomicOr(status, kSeedEnergy);
    return;
  }
  u.c[4][k] = adjusted;
  const double rho = u.c[0][k];
  if (!(isfinite(rho) && rho > 0.0)) {
    atomicOr(status, kSeedDensity);
    return;
  }
  const St st{rho, u.c[1][k], u.c[2][k], u.c[3][k], adjusted, bxc, byc, u.c[7][k]};
  const double p = pressure(st, gamma);
  if (!isfinite(p)) {
    atomicOr(status, kSeedEnergy);
    return;
  }
  if (!(p > 0.0)) atomicOr(status, kSeedPressure);
}

// One side's ghost layers, fluid (parts 1) or field (parts 2)
// (mhd_boundary_hip.hip:66-218).
__global__ void k_abi_fill_side(Grid g, StateP u, int side, int mode, int parts) {
  const int axis = side / 2;
  const int lines = (axis == 0 ? g.ny : g.nx) + 2 * g.ng;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= g.ng * lines) return;
  fill_ghost(g, u, axis, (side & 1) == 0, mode, t / lines + 1, t % lines - g.ng, parts);
}

__device__ __forceinline__ void atomic_min_lanes(unsigned long long* dst, unsigned long long v) {
  const cg::coalesced_group grp = cg::coalesced_threads();
  const unsigned long long m = cg::reduce(grp, v, cg::less<unsigned long long>());
  if (grp.thread_rank() == 0) atomicMin(dst, m);
}

// Cell state with the high-order (coll 0) or two-face (coll 1) collocated
// in-plane field, formed from the face arrays (mhd_staggering.hpp:321-338).
template <int W>
__device__ __forceinline__ St abi_cell(const Grid& g, const StateP& u, int i, int j, int coll) {
  if (coll) return load_cell1(u, g, i, j);
  const long long k = g.idx(i, j);
  return St{u.c[0][k], u.c[1][k], u.c[2][k], u.c[3][k], u.c[4][k],
            face_to_cell<W>(u.c[5], (long long)g.idx(0, j), 1, i, -g.ng, g.nx + g.ng - 1),
            face_to_cell<W>(u.c[6], (long long)g.idx(i, 0), g.pitch, j, -g.ng, g.ny + g.ng - 1),
            u.c[7][k]};
}

// Admissible convex fraction with density and internal-energy floors
// (mhd_reduce.hip:143-209); *theta holds the bits of the running minimum.
template <int W>
__global__ void __launch_bounds__(256) k_abi_admissible(Grid g, StateP base, StateP cand,
                                                        double rho_floor, double q_floor,
                                                        int coll, unsigned long long* theta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const St a = abi_cell<W>(g, base, i, j, coll), b = abi_cell<W>(g, cand, i, j, coll);
  double local = 1.0;
  const double qa = convex_q(a, b, 0.0);
  if (!(a.rho > rho_floor) || !(qa > q_floor) || !isfinite(a.rho) || !isfinite(qa)) {
    local = 0.0;
  } else if (!(isfinite(b.rho) && isfinite(b.mx) && isfinite(b.my) && isfinite(b.mz) &&
               isfinite(b.E) && isfinite(b.bx) && isfinite(b.by) && isfinite(b.bz))) {
    local = 0.0;
  } else {
    double hi = 1.0;
    if (b.rho <= rho_floor) {
      const double den = a.rho - b.rho;
      hi = den > 0.0 ? (a.rho - rho_floor) / den : 0.0;
      hi = fmin(fmax(hi, 0.0), 1.0);
    }
    if (convex_q(a, b, hi) > q_floor) {
      local = hi;
    } else {
      double lo = 0.0;
      for (int it = 0; it < 56; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (convex_q(a, b, mid) > q_floor) lo = mid;
        else hi = mid;
      }
      local = lo;
    }
  }
  atomic_min_lanes(theta, dbits(local));
}

// Relative solenoidality of the interior cells: acc[0] residual, acc[1]
// scale maxima (bits).
__global__ void __launch_bounds__(256) k_abi_divb_relative(Grid g, StateP u, int solver_owned,
                                                           unsigned long long* acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  unsigned long long rb, sb;
  divb_cell(g, u, g.idx(i, j), solver_owned, rb, sb);
  atomic_max_lanes(acc, rb);
  atomic_max_lanes(acc + 1, sb);
}

// CFL rate 0.5 alpha / h of the face with high cell (i, j) normal to DIR, as
// the face-flux kernels form it: the face-average Riemann problem and, for
// MP5/MP7, every Gauss point before the first inadmissible one
// (mhd_reduce.hip:254-416).
template <int DIR, int ORDER>
__device__ double abi_face_rate(const Grid& g, const IfaceP& in, int i, int j, double gamma) {
  int si = i, sj = j;
  if (DIR == 0 && i == g.nx && g.bc[0] == 0 && g.bc[1] == 0) si = 0;
  if (DIR == 1 && j == g.ny && g.bc[2] == 0 && g.bc[3] == 0) sj = 0;
  const long long ks = g.idx(si, sj);
  const double h = DIR == 0 ? g.dx : g.dy;
  double rate = face_rate<DIR, ORDER>(iface(in, ks, true), iface(in, ks, false), gamma, h);
  if (ORDER != 5 && ORDER != 7) return rate;
  constexpr int H = ORDER == 5 ? 2 : 3, N = 2 * H + 1, Q = ORDER == 5 ? 3 : 4;
  const long long ts = DIR == 0 ? g.pitch : 1;
  for (int q = 0; q < Q; ++q) {
    double w[N];
#pragma unroll
    for (int t = 0; t < N; ++t) w[t] = point_w<ORDER>(q, t);
    double pl[8], pr[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      double sa[N], sb[N];
#pragma unroll
      for (int t = 0; t < N; ++t) {
        sa[t] = in.L[c][ks + (t - H) * ts];
        sb[t] = in.R[c][ks + (t - H) * ts];
      }
      pl[c] = wsum<N>(w, sa);
      pr[c] = wsum<N>(w, sb);
    }
    const St l{pl[0], pl[1], pl[2], pl[3], pl[4], pl[5], pl[6], pl[7]};
    const St r{pr[0], pr[1], pr[2], pr[3], pr[4], pr[5], pr[6], pr[7]};
    if (!point_admissible(l, gamma) || !point_admissible(r, gamma)) break;
    rate = fmax(rate, face_rate<DIR, ORDER>(l, r, gamma, h));
  }
  return rate;
}

template <int ORDER>
__global__ void __launch_bounds__(256) k_abi_cfl_rate(Grid g, IfaceP ix, IfaceP iy, double gamma,
                                                      unsigned long long* max_rate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const double r = (abi_face_rate<0, ORDER>(g, ix, i, j, gamma) +
                    abi_face_rate<0, ORDER>(g, ix, i + 1, j, gamma)) +
                   (abi_face_rate<1, ORDER>(g, iy, i, j, gamma) +
                    abi_face_rate<1, ORDER>(g, iy, i, j + 1, gamma));
  const double local = isfinite(r) ? fmax(0.0, r) : kInf;
  atomic_max_lanes(max_rate, dbits(local));
}

__global__ void k_abi_set_u64(unsigned long long* p, int n, unsigned long long v) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = v;
}

std::mutex g_abi_mu;
Ctl* g_abi_ctl_ptr[64] = {};

}  // namespace

cudaError_t abi_zero_ctl(Ctl** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_abi_mu);
  if (!g_abi_ctl_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_abi_zero_ctl);
    if (e != cudaSuccess) return e;
    g_abi_ctl_ptr[dev] = static_cast<Ctl*>(p);
  }
  *out = g_abi_ctl_ptr[dev];
  return cudaSuccess;
}

void launch_abi_flux_difference(const Grid& g, const FluxP& f, int dir, const FluxP& d,
                                cudaStream_t s) {
  k_abi_flux_difference<<<dim3(cdiv(g.nx, kBX), cdiv(g.ny, 8)), dim3(kBX, 8), 0, s>>>(g, f, dir, d);
}

void launch_abi_curl_rate(const Grid& g, const double* ez, double* dbx, double* dby,
                          cudaStream_t s) {
  k_abi_curl_rate<<<dim3(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 8)), dim3(kBX, 8), 0, s>>>(g, ez, dbx,
                                                                                       dby);
}

void launch_abi_rk_stage(const Grid& g, const StateP& out, const StateP& un, const StateP& us,
                         const FluxP& d, double a, double b, double c, cudaStream_t s) {
  k_abi_rk_stage<<<dim3(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 8)), dim3(kBX, 8), 0, s>>>(
      g, out, un, us, d, a, b, c);
}

void launch_abi_collocate(const Grid& g, int axis, const double* face, double* cell,
                          cudaStream_t s) {
  const dim3 grid(cdiv(g.nx + 2 * g.ng, kBX), cdiv(g.ny + 2 * g.ng, 8)), block(kBX, 8);
  if (g.ng == 2) k_abi_collocate<4><<<grid, block, 0, s>>>(g, axis, face, cell);
  else if (g.ng == 3) k_abi_collocate<6><<<grid, block, 0, s>>>(g, axis, face, cell);
  else k_abi_collocate<8><<<grid, block, 0, s>>>(g, axis, face, cell);
}

void launch_abi_seed(const Grid& g, const SeedSpec& spec, const StateP& out, double* raw,
                     int* status, cudaStream_t s) {
  const dim3 block(kBX, 8), grid(cdiv(g.nx + 2 * g.ng, kBX), cdiv(g.ny + 2 * g.ng, 8));
  k_seed_pass1<<<grid, block, 0, s>>>(g, spec, out, raw, status);
  launch_abi_collocate(g, 0, out.c[5], out.bxc, s);
  launch_abi_collocate(g, 1, out.c[6], out.byc, s);
  k_seed_recollocate<<<grid, block, 0, s>>>(g, spec.gamma, out, raw, status);
}

void launch_abi_fill_side(const Grid& g, const StateP& u, int side, int mode, int parts,
                          cudaStream_t s) {
  const long long n = (long long)g.ng * ((side / 2 == 0 ? g.ny : g.nx) + 2 * g.ng);
  k_abi_fill_side<<<cdiv(n, 256), 256, 0, s>>>(g, u, side, mode, parts);
}

void launch_abi_admissible(const Grid& g, const StateP& base, const StateP& cand,
                           double rho_floor, double q_floor, int coll, unsigned long long* theta,
                           cudaStream_t s) {
  const dim3 grid(cdiv(g.nx, kBX), cdiv(g.ny, 8)), block(kBX, 8);
  if (g.ng == 2) k_abi_admissible<4><<<grid, block, 0, s>>>(g, base, cand, rho_floor, q_floor, coll, theta);
  else if (g.ng == 3) k_abi_admissible<6><<<grid, block, 0, s>>>(g, base, cand, rho_floor, q_floor, coll, theta);
  else k_abi_admissible<8><<<grid, block, 0, s>>>(g, base, cand, rho_floor, q_floor, coll, theta);
}

void launch_abi_divb_relative(const Grid& g, const StateP& u, int solver_owned,
                              unsigned long long* acc, cudaStream_t s) {
  k_abi_divb_relative<<<dim3(cdiv(g.nx, kBX), cdiv(g.ny, 8)), dim3(kBX, 8), 0, s>>>(
      g, u, solver_owned, acc);
}

void launch_abi_cfl_rate(const Grid& g, const IfaceP& ix, const IfaceP& iy, int order,
                         double gamma, unsigned long long* max_rate, cudaStream_t s) {
  const dim3 grid(cdiv(g.nx, kBX), cdiv(g.ny, 8)), block(kBX, 8);
  switch (order) {
    case 1: k_abi_cfl_rate<1><<<grid, block, 0, s>>>(g, ix, iy, gamma, max_rate); break;
    case 2: k_abi_cfl_rate<2><<<grid, block, 0, s>>>(g, ix, iy, gamma, max_rate); break;
    case 5: k_abi_cfl_rate<5><<<grid, block, 0, s>>>(g, ix, iy, gamma, max_rate); break;
    default: k_abi_cfl_rate<7><<<grid, block, 0, s>>>(g, ix, iy, gamma, max_rate);
  }
}

void launch_abi_set_u64(unsigned long long* p, int n, unsigned long long v, cudaStream_t s) {
  k_abi_set_u64<<<cdiv(n, 256), 256, 0, s>>>(p, n, v);
}

}  // namespace qb
