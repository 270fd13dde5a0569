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

namespace qb {

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
  return __ddiv_rn(__dadd_rn(lo_face, f[k + step]), 2.0);
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

// axis 0: the x sides (both), all padded rows; axis 1: the y sides over all
// padded columns (run after axis 0 so the corner blocks close last).
__global__ void k_fill_ghosts(Grid g, StateP u, int axis) {
  const int lines = (axis == 0 ? g.ny : g.nx) + 2 * g.ng;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 2 * g.ng * lines) return;
  const int side = t / (g.ng * lines);
  const int rem = t - side * g.ng * lines;
  const int layer = rem / lines + 1;
  const int line = rem % lines - g.ng;
  const bool lo = side == 0;
  const int mode = g.bc[axis * 2 + side];
  const int n = axis == 0 ? g.nx : g.ny;
  int gi, si;
  ghost_src(n, layer, lo, mode, gi, si);
  auto at = [&](int a) { return axis == 0 ? g.idx(a, line) : g.idx(line, a); };
  const long long kd = at(gi), ks = at(si);
  const double sn = mode == 2 ? -1.0 : 1.0;
  // fluid: the wall flips only the normal momentum
  u.c[0][kd] = u.c[0][ks];
  u.c[1][kd] = (axis == 0 ? sn : 1.0) * u.c[1][ks];
  u.c[2][kd] = (axis == 1 ? sn : 1.0) * u.c[2][ks];
  u.c[3][kd] = u.c[3][ks];
  u.c[4][kd] = u.c[4][ks];
  // field: tangential face and bz even; the normal face follows its own rule
  double* bn = axis == 0 ? u.c[5] : u.c[6];
  double* bt = axis == 0 ? u.c[6] : u.c[5];
  bt[kd] = bt[ks];
  u.c[7][kd] = u.c[7][ks];
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
__device__ double admissible_fraction(const St& a, const St& b) {
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

// Collocate the candidate state's in-plane field (padded range) and, for
// interior cells, run the admissibility fraction against `base` and the
// live-state preflights.  theta_mask: bit0 collocation order 0, bit1 order 1,
// bit2 order 1 only when the live state's low-order anchor is admissible.
template <int W>
__global__ void k_colloc_check(Grid g, StateP cand, StateP base, int has_base, int theta_mask,
                               int live_checks, int solver_owned, double gamma, Ctl* ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - g.ng;
  const int j = blockIdx.y * blockDim.y + threadIdx.y - g.ng;
  if (i >= g.nx + g.ng || j >= g.ny + g.ng) return;
  if (ctl->status & ~kStatusDone) return;
  const long long k = g.idx(i, j);
  const double bxc = face_to_cell<W>(cand.c[5], (long long)g.idx(0, j) - 0, 1, i, -g.ng,
                                     g.nx + g.ng - 1);
  const double byc = face_to_cell<W>(cand.c[6], (long long)g.idx(i, 0), g.pitch, j, -g.ng,
                                     g.ny + g.ng - 1);
  cand.bxc[k] = bxc;
  cand.byc[k] = byc;
  if (i < 0 || j < 0 || i >= g.nx || j >= g.ny) return;
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
    // discrete div B relative to the directional scale
    // (mhd_reduce.hip:556-700, solver mhd_solver.cpp:1196-1222)
    const double bxl = cand.c[5][k], bxh = cand.c[5][k + 1];
    const double byl = cand.c[6][k], byh = cand.c[6][k + g.pitch];
    const double d1 = __ddiv_rn(__dadd_rn(bxh, -bxl), g.dx);
    const double d2 = __ddiv_rn(__dadd_rn(byh, -byl), g.dy);
    const double res = __dadd_rn(d1, d2);
    const double scale = __dadd_rn(fabs(d1), fabs(d2));
    const double unc = __dadd_rn(__ddiv_rn(__dadd_rn(ulp_of(bxh), ulp_of(bxl)), g.dx),
                                 __ddiv_rn(__dadd_rn(ulp_of(byh), ulp_of(byl)), g.dy));
    bool explained;
    if (solver_owned) {
      explained = fabs(res) <= 1024.0 * unc;
    } else {
      explained = d1 != 0.0 && d2 != 0.0 && (signbit(d1) != signbit(d2)) &&
                  fabs(res) <= 0.5 * scale && fabs(res) <= 1024.0 * unc;
    }
    const double r = explained ? 0.0 : fabs(res);
    if (!isfinite(r) || !isfinite(scale)) {
      atomicMax(&ctl->divb_res, dbits(kInf));
    } else {
      if (r > 0.0) atomicMax(&ctl->divb_res, dbits(r));
      if (scale > 0.0) atomicMax(&ctl->divb_scale, dbits(scale));
    }
  }
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

// Conserved-variable 7-wave eigenvectors about `s` (x-normal), built as
// L = Lp dW/dU and R = dU/dW Rp with the reference's biorthogonality
// fallback to the identity (numerics/mhd_eigensystem.hpp:58-431).
// L row-major (waves x vars), R stored R[var*7 + wave].
__device__ void build_eig(const St& s, double gamma, double* L, double* R) {
  const Pr w = to_prim(s, gamma);
  const double rho = w.rho;
  const double p = w.p > 0.0 ? w.p : 0.0;
  const double sr = sqrt(rho);
  const double bn = w.bx, bt1 = w.by, bt2 = w.bz;
  double cf, cs, a, cax, ca;
  magnetosonic(rho, p, bn, bt1, bt2, gamma, cf, cs, a, cax, ca);
  double af, as;
  {
    // contraction-free: af2/as2 are differences of nearly equal squares at a
    // degenerate fan (mhd_eigensystem.hpp:91-110)
    const double sc = cf > 0.0 ? cf : 1.0;
    const double cfn = cf / sc, csn = cs / sc, an = a / sc;
    const double den = sub(mul(cfn, cfn), mul(csn, csn));
    if (den <= mul(64.0 * kEps, add(mul(cfn, cfn), mul(csn, csn)))) {
      af = 1.0 / sqrt(2.0);
      as = 1.0 / sqrt(2.0);
    } else {
      double af2 = sub(mul(an, an), mul(csn, csn)) / den;
      double as2 = sub(mul(cfn, cfn), mul(an, an)) / den;
      af = sqrt(af2 < 0.0 ? 0.0 : af2);
      as = sqrt(as2 < 0.0 ? 0.0 : as2);
    }
  }
  double b1, b2;
  {
    const double bt = scaled_norm3(bt1, bt2, 0.0);
    const double fs = a > ca ? a : ca;
    if (bt == 0.0 || bt / sr <= 64.0 * kEps * (fs + kTiny)) {
      b1 = 1.0 / sqrt(2.0);
      b2 = 1.0 / sqrt(2.0);
    } else {
      b1 = bt1 / bt;
      b2 = bt2 / bt;
    }
  }
  const double sbn = bn >= 0.0 ? 1.0 : -1.0;
  const double vn = w.vx, vt1 = w.vy, vt2 = w.vz;
  const double qf = cf * af * sbn, qs = cs * as * sbn;
  const double Af = a * af * sr, As = a * as * sr;
  const double ia2 = a > 0.0 ? (1.0 / a) / a : 0.0;
  const double Nf = 0.5 * ia2;
  const double ra2 = gamma * p;
  const double s2 = 1.0 / sqrt(2.0);
  double Rp[7][7], Lp[7][7];
#pragma unroll
  for (int k = 0; k < 7; ++k)
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      Rp[k][v] = 0.0;
      Lp[k][v] = 0.0;
    }
  Rp[0][0] = rho * af; Rp[0][1] = -af * cf; Rp[0][2] = qs * b1; Rp[0][3] = qs * b2;
  Rp[0][4] = af * ra2; Rp[0][5] = As * b1; Rp[0][6] = As * b2;
  Rp[6][0] = rho * af; Rp[6][1] = af * cf; Rp[6][2] = -qs * b1; Rp[6][3] = -qs * b2;
  Rp[6][4] = af * ra2; Rp[6][5] = As * b1; Rp[6][6] = As * b2;
  Rp[1][2] = -b2 * s2; Rp[1][3] = b1 * s2;
  Rp[1][5] = -sbn * b2 * s2 * sr; Rp[1][6] = sbn * b1 * s2 * sr;
  Rp[5][2] = -b2 * s2; Rp[5][3] = b1 * s2;
  Rp[5][5] = sbn * b2 * s2 * sr; Rp[5][6] = -sbn * b1 * s2 * sr;
  Rp[2][0] = rho * as; Rp[2][1] = -as * cs; Rp[2][2] = -qf * b1; Rp[2][3] = -qf * b2;
  Rp[2][4] = as * ra2; Rp[2][5] = -Af * b1; Rp[2][6] = -Af * b2;
  Rp[4][0] = rho * as; Rp[4][1] = as * cs; Rp[4][2] = qf * b1; Rp[4][3] = qf * b2;
  Rp[4][4] = as * ra2; Rp[4][5] = -Af * b1; Rp[4][6] = -Af * b2;
  Rp[3][0] = 1.0;
  Lp[0][1] = -Nf * af * cf; Lp[0][2] = Nf * qs * b1; Lp[0][3] = Nf * qs * b2;
  Lp[0][4] = Nf * af / rho; Lp[0][5] = Nf * As * b1 / rho; Lp[0][6] = Nf * As * b2 / rho;
  Lp[6][1] = Nf * af * cf; Lp[6][2] = -Nf * qs * b1; Lp[6][3] = -Nf * qs * b2;
  Lp[6][4] = Nf * af / rho; Lp[6][5] = Nf * As * b1 / rho; Lp[6][6] = Nf * As * b2 / rho;
  Lp[1][2] = -b2 * s2; Lp[1][3] = b1 * s2;
  Lp[1][5] = -sbn * b2 * s2 / sr; Lp[1][6] = sbn * b1 * s2 / sr;
  Lp[5][2] = -b2 * s2; Lp[5][3] = b1 * s2;
  Lp[5][5] = sbn * b2 * s2 / sr; Lp[5][6] = -sbn * b1 * s2 / sr;
  Lp[2][1] = -Nf * as * cs; Lp[2][2] = -Nf * qf * b1; Lp[2][3] = -Nf * qf * b2;
  Lp[2][4] = Nf * as / rho; Lp[2][5] = -Nf * Af * b1 / rho; Lp[2][6] = -Nf * Af * b2 / rho;
  Lp[4][1] = Nf * as * cs; Lp[4][2] = Nf * qf * b1; Lp[4][3] = Nf * qf * b2;
  Lp[4][4] = Nf * as / rho; Lp[4][5] = -Nf * Af * b1 / rho; Lp[4][6] = -Nf * Af * b2 / rho;
  Lp[3][0] = 1.0; Lp[3][4] = -ia2;
  // M = dU/dW and its analytic inverse, written as their non-zero pattern.
  const double gm1 = gamma - 1.0;
  const double hv2 = half_sq3(vn, vt1, vt2);
  const double ir = 1.0 / rho;
  const double Mi0[5] = {1.0, -vn * ir, -vt1 * ir, -vt2 * ir, gm1 * hv2};  // column 0, rows 0..4
  const double Mi4[7] = {gm1 * hv2, -gm1 * vn, -gm1 * vt1, -gm1 * vt2, gm1, -gm1 * bt1, -gm1 * bt2};
  const double Mdiag[7] = {1.0, ir, ir, ir, gm1, 1.0, 1.0};
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    // L[k][v] = sum_j Lp[k][j] Minv[j][v]   (j ascending, zeros skipped)
    double l0 = 0.0;
#pragma unroll
    for (int j = 0; j < 5; ++j) l0 += Lp[k][j] * Mi0[j];
    L[k * 7 + 0] = l0;
#pragma unroll
    for (int v = 1; v < 7; ++v) {
      double acc = Lp[k][v] * (v == 4 ? Mi4[4] : Mdiag[v]);
      if (v < 4) acc = acc + Lp[k][4] * Mi4[v];
      if (v > 4) acc = Lp[k][4] * Mi4[v] + Lp[k][v] * Mdiag[v];
      L[k * 7 + v] = acc;
    }
    // R[v][k] = sum_j M[v][j] Rp[k][j]
    R[0 * 7 + k] = Rp[k][0];
    R[1 * 7 + k] = vn * Rp[k][0] + rho * Rp[k][1];
    R[2 * 7 + k] = vt1 * Rp[k][0] + rho * Rp[k][2];
    R[3 * 7 + k] = vt2 * Rp[k][0] + rho * Rp[k][3];
    R[4 * 7 + k] = (((((hv2 * Rp[k][0] + (rho * vn) * Rp[k][1]) + (rho * vt1) * Rp[k][2]) +
                      (rho * vt2) * Rp[k][3]) + (1.0 / gm1) * Rp[k][4]) + bt1 * Rp[k][5]) +
                   bt2 * Rp[k][6];
    R[5 * 7 + k] = Rp[k][5];
    R[6 * 7 + k] = Rp[k][6];
  }
  bool usable = true;
  for (int i = 0; i < 7 && usable; ++i)
    for (int jj = 0; jj < 7; ++jj) {
      double dot = 0.0;
#pragma unroll
      for (int k = 0; k < 7; ++k) dot += L[i * 7 + k] * R[k * 7 + jj];
      const double expect = i == jj ? 1.0 : 0.0;
      if (!isfinite(dot) || fabs(dot - expect) > 1024.0 * kEps) {
        usable = false;
        break;
      }
    }
  if (!usable) {
#pragma unroll
    for (int e = 0; e < 49; ++e) {
      L[e] = (e % 8 == 0) ? 1.0 : 0.0;
      R[e] = (e % 8 == 0) ? 1.0 : 0.0;
    }
  }
}

// MP5 (H=2) / MP7 (H=3) characteristic L and R states at the face between
// cells k0-step and k0 (mhd_reconstruct.hip:217-349, 525-616).
template <int DIR, int H>
__device__ void mp_pair(const StateP& u, long long k0, long long step, double gamma, St& ul,
                        St& ur) {
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
  double L[49], R[49];
  build_eig(c, gamma, L, R);
  double ch[S][7];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const St d = rot<DIR>(load_cell(u, k0 + (long long)(s - 1 - H) * step));
    const double u7[7] = {d.rho - c.rho, d.mx - c.mx, d.my - c.my, d.mz - c.mz,
                          d.E - c.E,     d.by - c.by, d.bz - c.bz};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      double acc = 0.0;
#pragma unroll
      for (int v = 0; v < 7; ++v) acc += L[k * 7 + v] * u7[v];
      ch[s][k] = acc;
    }
  }
  double dl[7], dr[7];
#pragma unroll
  for (int v = 0; v < 7; ++v) {
    dl[v] = 0.0;
    dr[v] = 0.0;
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    double win[W];
    bool f;
#pragma unroll
    for (int s = 0; s < W; ++s) win[s] = ch[s][k];
    const double wl = mp_recon<W>(win, f);
#pragma unroll
    for (int s = 0; s < W; ++s) win[s] = ch[W - s][k];
    const double wr = mp_recon<W>(win, f);
#pragma unroll
    for (int v = 0; v < 7; ++v) {
      dl[v] += R[v * 7 + k] * wl;
      dr[v] += R[v * 7 + k] * wr;
    }
  }
  const St sl{c.rho + dl[0], c.mx + dl[1], c.my + dl[2], c.mz + dl[3],
              c.E + dl[4],   c.bx,         c.by + dl[5], c.bz + dl[6]};
  const St sr{c.rho + dr[0], c.mx + dr[1], c.my + dr[2], c.mz + dr[3],
              c.E + dr[4],   c.bx,         c.by + dr[5], c.bz + dr[6]};
  ul = rot<DIR>(sl);
  ur = rot<DIR>(sr);
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

template <int DIR, int ORDER>
__global__ void __launch_bounds__(128) k_reconstruct(Grid g, StateP u, IfaceP out, double gamma,
                                                     const Ctl* ctl) {
  // dir 0: faces i in [0,nx] over all padded rows; dir 1: transposed.
  const int i = blockIdx.x * blockDim.x + threadIdx.x - (DIR == 1 ? g.ng : 0);
  const int j = blockIdx.y * blockDim.y + threadIdx.y - (DIR == 0 ? g.ng : 0);
  if (DIR == 0 ? (i > g.nx || j >= g.ny + g.ng) : (i >= g.nx + g.ng || j > g.ny)) return;
  if (ctl->status & ~kStatusDone) return;
  const long long k0 = g.idx(i, j);
  const long long step = DIR == 0 ? 1 : g.pitch;
  St ul, ur;
  if (ORDER <= 1) {
    ul = DIR == 0 ? load_cell1(u, g, i - 1, j) : load_cell1(u, g, i, j - 1);
    ur = load_cell1(u, g, i, j);
  } else if (ORDER == 2) {
    muscl_pair<DIR>(g, u, i, j, k0, step, gamma, ul, ur);
  } else {
    mp_pair<DIR, ORDER == 5 ? 2 : 3>(u, k0, step, gamma, ul, ur);
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

// One side's |v_n| and fast speed (mhd_reduce.hip:254-325).
template <int DIR>
__device__ Spd speed_parts(const St& s, double gamma) {
  const double p = pressure(s, gamma);
  if (!(isfinite(s.rho) && s.rho > 0.0 && isfinite(s.mx) && isfinite(s.my) &&
        isfinite(s.mz) && isfinite(s.E) && isfinite(s.bx) && isfinite(s.by) &&
        isfinite(s.bz) && isfinite(p) && p > 0.0))
    return Spd{kInf, kInf};
  const double sr = sqrt(s.rho);
  const double sound = mul(sqrt(gamma), sqrt(p)) / sr;
  const double ax = s.bx / sr, ay = s.by / sr, az = s.bz / sr;
  if (!(isfinite(sound) && isfinite(ax) && isfinite(ay) && isfinite(az))) return Spd{kInf, kInf};
  const double ca = scaled_norm3(ax, ay, az);
  const double can = fabs(DIR == 0 ? ax : ay);
  const double scale = fmax(sound, ca);
  double fast = 0.0;
  if (scale > 0.0) {
    const double an = sound / scale, bn = ca / scale, cn = can / scale;
    const double a2 = mul(an, an), b2 = mul(bn, bn), sum = add(a2, b2);
    double disc = sub(mul(sum, sum), mul(mul(mul(4.0, a2), cn), cn));
    if (disc < 0.0) disc = 0.0;
    fast = mul(scale, sqrt(mul(0.5, add(sum, sqrt(disc)))));
  }
  const double vel = fabs(DIR == 0 ? s.mx : s.my) / s.rho;
  if (!(isfinite(vel) && isfinite(fast))) return Spd{kInf, kInf};
  return Spd{vel, fast};
}

// Weighted face rate 0.5*alpha/h of one Riemann problem (mhd_reduce.hip:331-383).
template <int DIR, int ORDER>
__device__ __forceinline__ double face_rate(const St& l, const St& r, double gamma, double h) {
  const Spd a = speed_parts<DIR>(l, gamma), b = speed_parts<DIR>(r, gamma);
  const double rate = ORDER <= 1 ? fmax(a.v + a.f, b.v + b.f) : fmax(a.v, b.v) + fmax(a.f, b.f);
  if (!(isfinite(rate) && rate >= 0.0)) return kInf;
  return (rate * 0.5) / h;
}

__device__ __forceinline__ St iface(const IfaceP& v, long long k, bool left) {
  double* const* a = left ? v.L : v.R;
  return St{__ldg(a[0] + k), __ldg(a[1] + k), __ldg(a[2] + k), __ldg(a[3] + k),
            __ldg(a[4] + k), __ldg(a[5] + k), __ldg(a[6] + k), __ldg(a[7] + k)};
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
  out.f[0][k] = f.rho;
  out.f[1][k] = f.mx;
  out.f[2][k] = f.my;
  out.f[3][k] = f.mz;
  out.f[4][k] = f.E;
  out.f[5][k] = f.bx;
  out.f[6][k] = f.by;
  out.f[7][k] = f.bz;
  // Directional Godunov E_z: F_x(By) = -Ez, F_y(Bx) = +Ez (mhd_ct.hip:126-133).
  emf[k] = DIR == 0 ? -f.by : f.bx;
  if (spd) spd[k] = rate;
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

// ===========================================================================
// Constrained transport and the stage update
// ===========================================================================
namespace {

// E_z = -(v x B)_z (mhd_ct.hip:408-417, zero background)
__device__ __forceinline__ double physical_ez(const St& s) {
  const double vx = s.mx / s.rho, vy = s.my / s.rho;
  return __dadd_rn(__dmul_rn(vy, s.bx), __dmul_rn(vx, -s.by));
}

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
          if (!point_admissible(p, gamma)) ok = false;
          pt[qy][qx] = physical_ez(p);
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
  if (i < g.nx && j < g.ny) {
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

// Face -> edge interpolation (mhd_ct.hip:50-97) with the constant shortcut.
template <int NT>
__device__ __forceinline__ double edge_interp(const double* e) {
  bool same = true;
#pragma unroll
  for (int q = 1; q < NT; ++q) same = same && (e[q] == e[0]);
  if (same) return e[0];
  if (NT == 2) return __ddiv_rn(__dadd_rn(e[0], e[1]), 2.0);
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

// Flux difference + EMF curl + Shu-Osher combine (mhd_update.hip:21-206,
// mhd_ct.hip:893-931, mhd_solver.cpp:840-874).  Writes cells and the owned
// high faces of the output; ghosts are closed by fill_ghosts afterwards.
__global__ void __launch_bounds__(256) k_update(Grid g, StateP un, StateP us, StateP out,
                                                FluxP fx, FluxP fy, const double* ez,
                                                const double* dt_dev, double dt_host, int stage,
                                                const Ctl* ctl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
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
  if (i < g.nx && j < g.ny) {
    const int cc[6] = {0, 1, 2, 3, 4, 7};
#pragma unroll
    for (int t = 0; t < 6; ++t) {
      const int q = cc[t];
      const double dqx = __dadd_rn(__ddiv_rn(fx.f[q][k + 1], g.dx), __ddiv_rn(-fx.f[q][k], g.dx));
      const double dqy =
          __dadd_rn(__ddiv_rn(fy.f[q][k + g.pitch], g.dy), __ddiv_rn(-fy.f[q][k], g.dy));
      const double d = __dadd_rn(-dqx, -dqy);
      out.c[q][k] = combine(un.c[q][k], b == 0.0 ? 0.0 : us.c[q][k], d);
    }
  }
  if (j < g.ny) {
    const double d = __dadd_rn(__ddiv_rn(-ez[k + g.pitch], g.dy), __ddiv_rn(ez[k], g.dy));
    out.c[5][k] = combine(un.c[5][k], b == 0.0 ? 0.0 : us.c[5][k], d);
  }
  if (i < g.nx) {
    const double d = __dadd_rn(__ddiv_rn(ez[k + 1], g.dx), __ddiv_rn(-ez[k], g.dx));
    out.c[6][k] = combine(un.c[6][k], b == 0.0 ? 0.0 : us.c[6][k], d);
  }
}

// Consume the live-state preflights computed with the previous state and
// reset the per-step reductions.  coll selects which collocation the
// admissibility preflight uses (mhd_solver.cpp:689-692); anchor_mode >= 0
// forces the low-order anchor flag, -1 derives it from the live state.
__global__ void k_step_begin(Ctl* ctl, int coll, int anchor_mode) {
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

// Clear the status word and the live-state accumulators before the live
// state's preflights are recomputed.
__global__ void k_reset_stats(Ctl* ctl) {
  ctl->status = 0;
  ctl->live_theta = dbits(1.0);
  ctl->anchor_theta = dbits(1.0);
  ctl->divb_res = 0ull;
  ctl->divb_scale = 0ull;
}

__global__ void k_set_time(Ctl* ctl, double t, double t_end) {
  ctl->t = t;
  ctl->t_end = t_end;
  ctl->steps_done = 0;
  ctl->status = 0;
}

// dt = cfl_eff / max_rate (mhd_solver.cpp:1283-1320), optionally clipped to
// the remaining interval of a device-resident run.
__global__ void k_dt(Ctl* ctl, double cfl_eff, double hmin, double hmax, int clip) {
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

__global__ void k_step_end(Ctl* ctl) {
  if (ctl->status) return;
  const double rem = ctl->t_end - ctl->t;
  ctl->t = ctl->dt == rem ? ctl->t_end : ctl->t + ctl->dt;
  ctl->steps_done += 1;
  if (!(ctl->t < ctl->t_end)) ctl->status |= kStatusDone;
}

__global__ void k_divb_linf(Grid g, StateP u, unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const long long k = g.idx(i, j);
  // ct_divb_linf_kernel (mhd_reduce.hip:505-553)
  const double d = __dadd_rn(__dadd_rn(__ddiv_rn(u.c[5][k + 1], g.dx), __ddiv_rn(-u.c[5][k], g.dx)),
                             __dadd_rn(__ddiv_rn(u.c[6][k + g.pitch], g.dy),
                                       __ddiv_rn(-u.c[6][k], g.dy)));
  const double v = isfinite(d) ? fabs(d) : kInf;
  if (v > 0.0) atomicMax(out, dbits(v));
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
// Launch wrappers
// ===========================================================================
namespace {
inline unsigned cdiv(long long a, int b) { return unsigned((a + b - 1) / b); }
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
  k_reconstruct<DIR, ORDER><<<grid, block, 0, s>>>(g, a.u, DIR == 0 ? a.ix : a.iy, a.gamma, a.ctl);
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

void launch_cell_emf(const StageArgs& a, bool cfl_reduce, cudaStream_t s) {
  const Grid& g = a.g;
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

void launch_corner_emf(const StageArgs& a, cudaStream_t s) {
  const Grid& g = a.g;
  const dim3 block(kBX, 4);
  const dim3 grid(cdiv(g.nx + 1, kBX), cdiv(g.ny + 1, 4));
  switch (a.order) {
    case 1:
    case 2: k_corner_emf<2><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl); break;
    case 5: k_corner_emf<5><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl); break;
    default: k_corner_emf<7><<<grid, block, 0, s>>>(g, a.cell_ez, a.xemf, a.yemf, a.xnj, a.ynj, a.ez, a.ctl);
  }
}

void launch_update(const StageArgs& a, const StateP& un, const StateP& us, const StateP& out,
                   int stage, const double* dt_dev, double dt_host, cudaStream_t s) {
  const Grid& g = a.g;
  const dim3 block(kBX, 8);
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

}  // namespace qb
