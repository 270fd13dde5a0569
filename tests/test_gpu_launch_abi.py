"""The per-kernel launch interface (include/quasar_mhd_launch.h, the C ABI of
the reference's backend seam include/quasar/physics/mhd/kernels.hpp) on the
GPU.  An SSP-RK3 step composed from the launch calls in the reference
solver's order (residual: mhd_solver.cpp:680-800; stage combine:
mhd_solver.cpp:853-874, ssprk_integrator.cpp:40-53) reproduces the solver's
own fused step bit for bit, and the standalone reductions agree with the
solver's."""
import numpy as np
import pytest

import mhd_cases as M

pytestmark = pytest.mark.gpu

ORDER_NAME = {2: "muscl_minmod", 5: "mp5", 7: "mp7"}
BC_NAME = {0: "periodic", 1: "outflow", 2: "wall"}
WALL = (2, 2, 2, 2)
# the wall case needs a field with no normal component at the walls: a
# field-free blast (pressure ratio 10)
CASES = [("ot", 48, 5, M.PERIODIC), ("rotor", 40, 7, M.OUTFLOW), ("blast", 36, 5, WALL),
         ("ot", 32, 2, M.PERIODIC)]
GENERATORS = {"ot": M.orszag_tang, "rotor": M.rotor,
              "blast": lambda n, order: M.blast(n, order=order, p_in=10.0, p_out=1.0, b=0.0)}
GAMMA = 5.0 / 3.0


def solver(n, order, bc):
    from quasar_b200 import mhd
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(n, n, 1.0, 1.0)
    cfg.reconstruction = ORDER_NAME[order]
    cfg.gamma = GAMMA
    cfg.boundary = mhd.MhdBoundarySpec([BC_NAME[b] for b in bc], [BC_NAME[b] for b in bc])
    s = mhd.MhdSolver2D(cfg)
    for name, a in zip(M.COMPONENTS, GENERATORS[CASE_OF[(n, order, bc)]](n, order=order)):
        s.seed_state(name, a)
    return s


CASE_OF = {(n, order, bc): case for case, n, order, bc in CASES}


class Workspace:
    """Caller-owned device buffers of one grid, as the reference solver owns
    them: registers, residual, fluxes, interface states, EMF tables."""

    def __init__(self, n, order):
        import torch
        from quasar_b200 import launch as L
        self.L, self.torch = L, torch
        ng = M.nghost(order)
        self.size = (n + 2 * ng) ** 2
        self.grid = L.Grid(n, n, ng, 1.0 / n, 1.0 / n)
        dev = torch.device("cuda")
        arr = lambda dt=torch.float64: torch.zeros(self.size, dtype=dt, device=dev)  # noqa: E731
        self.regs = [[arr() for _ in range(8)] for _ in range(2)]
        self.dudt = [arr() for _ in range(8)]
        self.fx = [arr() for _ in range(8)]
        self.fy = [arr() for _ in range(8)]
        self.ix = ([arr() for _ in range(8)], [arr() for _ in range(8)])
        self.iy = ([arr() for _ in range(8)], [arr() for _ in range(8)])
        self.cbx, self.cby = arr(), arr()
        self.emf_arrays = (arr(), arr(), arr(torch.int32), arr(torch.int32), arr(), arr())
        self.scratch = torch.zeros(8, dtype=torch.float64, device=dev)
        self.dev = dev

    def upload(self, s):
        return [self.torch.from_numpy(s.state_component_to_host(c)).to(self.dev)
                for c in M.COMPONENTS]

    def interfaces(self, u, order, bc):
        L = self.L
        fl = L.flags(bc)
        ifx, ify = L.iface(*self.ix), L.iface(*self.iy)
        L.reconstruct(self.grid, L.field(u), self.cbx, self.cby, 0, ifx, order, fl, GAMMA)
        L.reconstruct(self.grid, L.field(u), self.cbx, self.cby, 1, ify, order, fl, GAMMA)
        return ifx, ify

    def step(self, u0, order, bc, dt):
        L = self.L
        fl = L.flags(bc)
        table = L.emf(*self.emf_arrays)
        U0, D = L.field(u0), L.field(self.dudt)
        us = u0
        for st, (a, b, c) in enumerate([(1.0, 0.0, 1.0), (3.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0),
                                        (1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0)]):
            Us = L.field(us)
            L.fill_ghosts(self.grid, Us, bc)
            for t in self.dudt:
                t.zero_()
            ifx, ify = L.iface(*self.ix), L.iface(*self.iy)
            L.reconstruct(self.grid, Us, self.cbx, self.cby, 0, ifx, order, fl, GAMMA)
            L.hlld_flux(self.grid, ifx, 0, L.field(self.fx), fl, GAMMA, order)
            L.reconstruct(self.grid, Us, self.cbx, self.cby, 1, ify, order, fl, GAMMA)
            L.hlld_flux(self.grid, ify, 1, L.field(self.fy), fl, GAMMA, order)
            L.flux_difference(self.grid, L.field(self.fx), 0, D)
            L.flux_difference(self.grid, L.field(self.fy), 1, D)
            L.ct_emf_prepare(self.grid, Us, self.cbx, self.cby, ifx, ify, fl, table, GAMMA, order)
            L.ct_emf_finish(self.grid, fl, table, order)
            L.emf_curl_rate(self.grid, table, D)
            out = self.regs[st % 2]
            L.rk_stage(self.grid, L.field(out), U0, Us, D, a, b, c * dt)
            us = out
        L.fill_ghosts(self.grid, L.field(us), bc)
        self.torch.cuda.synchronize()
        return [t.cpu().numpy() for t in us]


@pytest.mark.parametrize("case,n,order,bc", CASES)
def test_composed_step_matches_solver_step(case, n, order, bc):
    s = solver(n, order, bc)
    w = Workspace(n, order)
    u0 = w.upload(s)
    dt = s.cfl_limit()
    got = w.step(u0, order, bc, dt)
    s.step_unchecked(dt)
    assert s.last_positivity_substeps() == 1
    want = [s.state_component_to_host(c) for c in M.COMPONENTS]
    for c, g, e in zip(M.COMPONENTS, got, want):
        diff = np.abs(g - e)
        assert np.array_equal(g, e), (c, float(np.nanmax(diff)), int(np.nanargmax(diff)))


@pytest.mark.parametrize("case,n,order,bc", CASES)
def test_reductions_match_solver(case, n, order, bc):
    s = solver(n, order, bc)
    w = Workspace(n, order)
    L = w.L
    u0 = w.upload(s)
    U0 = L.field(u0)
    L.fill_ghosts(w.grid, U0, bc)
    ifx, ify = w.interfaces(u0, order, bc)
    rate = L.cfl_max_rate(w.grid, ifx, ify, GAMMA, w.scratch, order, L.flags(bc))
    assert rate.rate_scale == 1.0
    cfl_eff = min(0.4, 0.2) if order >= 5 else 0.4
    assert cfl_eff / rate.scaled_max_rate == s.cfl_limit()
    assert L.ct_divb_linf(w.grid, U0, w.scratch) == s.divergence_b_max()
    assert L.ct_divb_relative_linf(w.grid, U0, w.scratch) <= 1024 * np.finfo(float).eps
    # the launch form sums 8192-cell chunks on the device, the solver's
    # totals finish its block partials on the host: two summation orders of
    # compensated sums, equal to a few ulp
    for got, want in zip(L.conserved_cell_sums(w.grid, U0), s.conserved_cell_totals()):
        assert abs(got - want) <= 1e-13 * abs(want), (got, want)
    assert L.admissible_fraction(w.grid, U0, U0, 0.0, 0.0, GAMMA, w.scratch) == 1.0
    # one cell of the candidate with its density negated: the edge of the
    # admissible segment is that cell's, found by the bisection restated here
    cand = [t.clone() for t in u0]
    ng = M.nghost(order)
    k = (n // 2 + ng) + (n + 2 * ng) * (n // 3 + ng)
    cand[0][k] = -cand[0][k]
    a = [float(u0[c][k]) for c in range(5)] + [
        float(s.state_component_to_host(c)[k]) for c in ("bx", "by")] + [float(u0[7][k])]
    b = [-a[0]] + a[1:]
    for rho_floor, p_floor in ((0.0, 0.0), (0.25 * a[0], 0.0), (0.0, 0.01)):
        th = L.admissible_fraction(w.grid, U0, L.field(cand), rho_floor, p_floor, GAMMA,
                                   w.scratch)
        want = expected_theta(a, b, rho_floor, p_floor / (GAMMA - 1.0))
        assert abs(th - want) <= 1e-9, (rho_floor, p_floor, th, want)
    th1 = L.admissible_fraction(w.grid, U0, L.field(cand), 0.0, 0.0, GAMMA, w.scratch, 1)
    assert 0.0 < th1 < 0.5


def expected_theta(a, b, rho_floor, q_floor):
    """Admissible convex fraction of one cell (mhd_reduce.hip:143-209) in
    plain float64: density bound, then 56 bisection steps on the internal
    energy."""
    def q(th):
        v = [(1.0 - th) * x + th * y for x, y in zip(a, b)]
        if not v[0] > 0.0:
            return -np.inf
        return (v[4] - 0.5 * (v[1] ** 2 + v[2] ** 2 + v[3] ** 2) / v[0]) - 0.5 * (
            v[5] ** 2 + v[6] ** 2 + v[7] ** 2)
    if not (a[0] > rho_floor and q(0.0) > q_floor):
        return 0.0
    hi = 1.0
    if b[0] <= rho_floor:
        hi = min(max((a[0] - rho_floor) / (a[0] - b[0]), 0.0), 1.0)
    if q(hi) > q_floor:
        return hi
    lo = 0.0
    for _ in range(56):
        mid = 0.5 * (lo + hi)
        if q(mid) > q_floor:
            lo = mid
        else:
            hi = mid
    return lo


def test_collocation_matches_solver_read():
    n, order, bc = 40, 7, M.OUTFLOW
    s = solver(n, order, bc)
    w = Workspace(n, order)
    u0 = w.upload(s)
    w.L.collocate_face_to_cell(w.grid, 0, u0[5], w.cbx)
    w.L.collocate_face_to_cell(w.grid, 1, u0[6], w.cby)
    w.torch.cuda.synchronize()
    ng = M.nghost(order)
    sl = (slice(ng, ng + n), slice(ng, ng + n))
    shape = (n + 2 * ng, n + 2 * ng)
    for got, name in ((w.cbx, "bx"), (w.cby, "by")):
        want = s.state_component_to_host(name).reshape(shape)[sl]
        assert np.array_equal(got.cpu().numpy().reshape(shape)[sl], want)
