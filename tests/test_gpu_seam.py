"""The reference's own, unmodified MhdSolver2D (mhd_solver.cpp with its
numerics registry) running on this project's kernels through the per-kernel
seam: oracle/seam/mhd_kernels_b200.cpp defines every kernels.hpp declaration
over include/quasar_mhd_launch.h, oracle/build_seam.sh links the result into
oracle/_ref/libquasar_mhd_seam.so with the same qref_* driver as the CPU
build.  The reference's host sequencing, interface cache, CFL path
(rate-only reconstruction), positivity controller, solenoidality preflight
and diagnostics all run unchanged; only the kernels are this project's.

Checks: against the reference built for the CPU (per-step state within 1e-10
relative L1 per physical group, dt within 1e-12 relative, same diagnostics
and the same error), and against this project's fused solver step (bit for
bit: the seam launches the same kernels in the reference's order)."""
import ctypes
import os

import numpy as np
import pytest

import mhd_cases as M

pytestmark = pytest.mark.gpu

SEAM_SO = os.path.join(M.ROOT, "oracle", "_ref", "libquasar_mhd_seam.so")
ORDER_NAME = {2: "muscl_minmod", 5: "mp5", 7: "mp7"}
BC_NAME = {0: "periodic", 1: "outflow", 2: "wall"}
STEP_TOL = 1e-10
DT_TOL = 1e-12


@pytest.fixture(scope="module")
def seam():
    if not os.path.exists(SEAM_SO):
        pytest.skip("seam build absent (oracle/build_seam.sh)")
    return M.RefLib(SEAM_SO)


def totals(lib, s):
    lib.lib.qref_totals.argtypes = [ctypes.c_void_p, M._dp, M._dp]
    m, e = ctypes.c_double(), ctypes.c_double()
    assert lib.lib.qref_totals(s.h, m, e) == 0, lib.err()
    return m.value, e.value


def divb(lib, s):
    d = ctypes.c_double()
    assert lib.lib.qref_divb(s.h, d) == 0, lib.err()
    return d.value


def fused(nx, ny, order, bc, lx=1.0, ly=1.0, ox=0.0, oy=0.0):
    from quasar_b200 import mhd
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(nx, ny, lx, ly, ox, oy)
    cfg.reconstruction = ORDER_NAME[order]
    cfg.boundary = mhd.MhdBoundarySpec([BC_NAME[b] for b in bc], [BC_NAME[b] for b in bc])
    return mhd.MhdSolver2D(cfg)


def pulse(nx, ny, order, bc, lx, ly, ox, oy):
    """Pressure pulse off centre, field tangential to every wall."""
    from quasar_b200 import ics
    ng = M.nghost(order)
    X, Y = np.meshgrid(ics._centres(nx, ng, lx, ox), ics._centres(ny, ng, ly, oy), indexing="xy")
    r = np.hypot(X - 0.3, Y - 0.55)
    p = np.where(r < 0.2, 5.0, 0.5)
    rho = 1.0 + 0.2 * np.exp(-8.0 * r * r)
    zero = np.zeros_like(X)
    by = zero + (0.6 if bc[2] != 2 and bc[3] != 2 else 0.0)
    return ics._assemble(rho, 0.1 * np.cos(2.0 * Y), zero, zero, p, zero, by, zero + 0.3, 5.0 / 3.0)


CASES = {
    "ot32_mp5": dict(n=(32, 32), order=5, bc=M.PERIODIC, ic=lambda: M.orszag_tang(32, order=5)),
    "rotor32_mp7": dict(n=(32, 32), order=7, bc=M.PERIODIC, ic=lambda: M.rotor(32, order=7)),
    "blast32_mp7": dict(n=(32, 32), order=7, bc=M.PERIODIC, ic=lambda: M.blast(32, order=7)),
    "pulse40x24_mp7_walls": dict(n=(40, 24), order=7, bc=(2, 2, 2, 2), dom=(2.0, 0.75, -1.0, 0.25)),
    "pulse40x24_mp5_mixed": dict(n=(40, 24), order=5, bc=(1, 2, 0, 0), dom=(2.0, 0.75, -1.0, 0.25)),
    "ot24_muscl": dict(n=(24, 24), order=2, bc=M.PERIODIC, ic=lambda: M.orszag_tang(24, order=2)),
}


def setup(case):
    c = CASES[case]
    nx, ny = c["n"]
    lx, ly, ox, oy = c.get("dom", (1.0, 1.0, 0.0, 0.0))
    ic = c["ic"]() if "ic" in c else pulse(nx, ny, c["order"], c["bc"], lx, ly, ox, oy)
    return nx, ny, c["order"], c["bc"], (lx, ly, ox, oy), ic


@pytest.mark.parametrize("case", list(CASES))
def test_reference_solver_on_seam_matches_cpu_reference(seam, ref, case):
    nx, ny, order, bc, (lx, ly, ox, oy), ic = setup(case)
    ng = M.nghost(order)
    g = seam.solver(nx, ny, order, bc=bc, lx=lx, ly=ly, ox=ox, oy=oy)
    c = ref.solver(nx, ny, order, bc=bc, lx=lx, ly=ly, ox=ox, oy=oy)
    g.seed(ic)
    c.seed(ic)
    for k in range(5):
        dt_c, dt_g = c.cfl(), g.cfl()
        assert abs(dt_g - dt_c) <= DT_TOL * dt_c, (k, dt_g, dt_c)
        c.step(dt_c)
        g.step(dt_c)
        assert g.substeps() == c.substeps()
        err = M.state_rel_l1(g.read(), c.read(), ng, nx, ny)
        assert err <= STEP_TOL, (k, err)
    assert divb(seam, g) <= 1e-12 and divb(ref, c) <= 1e-12
    (mg, eg), (mc, ec) = totals(seam, g), totals(ref, c)
    assert abs(mg - mc) <= 1e-12 * abs(mc)
    assert abs(eg - ec) <= 1e-12 * abs(ec)


@pytest.mark.parametrize("case", ["ot32_mp5", "rotor32_mp7", "pulse40x24_mp7_walls", "ot24_muscl"])
def test_reference_solver_on_seam_equals_fused_step(seam, case):
    """The reference's driver over the seam and this project's fused step
    launch the same kernels: dt and state agree bit for bit."""
    nx, ny, order, bc, (lx, ly, ox, oy), ic = setup(case)
    g = seam.solver(nx, ny, order, bc=bc, lx=lx, ly=ly, ox=ox, oy=oy)
    f = fused(nx, ny, order, bc, lx, ly, ox, oy)
    g.seed(ic)
    for name, a in zip(M.COMPONENTS, ic):
        f.seed_state(name, a)
    shape = g.shape
    for k in range(4):
        dt = g.cfl()
        assert f.cfl_limit() == dt, k
        g.step(dt)
        f.step_unchecked(dt)
        mine = [f.state_component_to_host(cn).reshape(shape) for cn in M.COMPONENTS]
        theirs = g.read()
        for c, (a, b) in enumerate(zip(mine, theirs)):
            np.testing.assert_array_equal(M._evolved(a, c, g.ng, nx, ny),
                                          M._evolved(b, c, g.ng, nx, ny),
                                          err_msg=f"step {k} {M.COMPONENTS[c]}")


def test_seam_raises_the_reference_preflight_error(seam, ref):
    """A face field that is not discretely solenoidal: the reference's
    preflight (its divb-relative launch, here this project's kernel) refuses
    the step with the same message on both builds."""
    nx = ny = 32
    ic = list(M.orszag_tang(32, order=5))
    rng = np.random.default_rng(3)
    ic[5] = ic[5] + 1e-3 * rng.standard_normal(ic[5].shape)
    msgs = []
    for lib in (seam, ref):
        s = lib.solver(nx, ny, 5)
        with pytest.raises(RuntimeError) as e:
            s.seed(ic)
            s.step(1e-4)
        msgs.append(str(e.value))
    assert "divergence-free" in msgs[0]
    assert msgs[0] == msgs[1]


def test_reference_positivity_controller_on_seam(seam, ref):
    """A step three times the CFL limit on a blast with a thousandfold core
    energy: the reference's controller rolls back and retries with smaller
    substeps and the order-1 anchor, calling this project's admissible-
    fraction and order-1 kernels.  Same substep count and state as the
    reference's CPU build; same as this project's fused controller."""
    n, order = 16, 5
    ic = list(M.blast(n, order=order))
    ic[4] = np.where(ic[4] > 100, ic[4] * 1e3, ic[4])
    g = seam.solver(n, n, order, bc=M.OUTFLOW)
    c = ref.solver(n, n, order, bc=M.OUTFLOW)
    f = fused(n, n, order, M.OUTFLOW)
    g.seed(ic)
    c.seed(ic)
    for name, a in zip(M.COMPONENTS, ic):
        f.seed_state(name, a)
    dt = 3.0 * c.cfl()
    c.step(dt)
    g.step(dt)
    f.step_unchecked(dt)
    assert g.substeps() == c.substeps() == f.last_positivity_substeps() >= 2
    mine = [f.state_component_to_host(cn).reshape(g.shape) for cn in M.COMPONENTS]
    assert M.state_rel_l1(g.read(), c.read(), g.ng, n, n) <= STEP_TOL
    assert M.state_rel_l1(mine, g.read(), g.ng, n, n) <= STEP_TOL


def test_exhausted_controller_matches_reference_driver(seam):
    """Blast 128^2 MP5 with outflow sides under the automatic dt: this
    project's fused solver and the reference's driver over the seam take the
    same dt and substeps and stay bit-identical for 60 steps (one of them
    with a positivity retry); on step 61 the controller runs out of
    representable time progress in both, with the reference's message and
    the same counters."""
    n, order = 128, 5
    ic = list(M.blast(n, order=order))
    g = seam.solver(n, n, order, bc=M.OUTFLOW)
    f = fused(n, n, order, M.OUTFLOW)
    g.seed(ic)
    for name, a in zip(M.COMPONENTS, ic):
        f.seed_state(name, a)
    retried = 0
    for k in range(61):
        dt = g.cfl()
        assert f.cfl_limit() == dt, k
        g.step(dt)
        f.step_unchecked(dt)
        assert g.substeps() == f.last_positivity_substeps(), k
        retried += g.substeps() > 1
    assert retried >= 1
    mine = [f.state_component_to_host(cn).reshape(g.shape) for cn in M.COMPONENTS]
    for c, (a, b) in enumerate(zip(mine, g.read())):
        np.testing.assert_array_equal(M._evolved(a, c, g.ng, n, n), M._evolved(b, c, g.ng, n, n))
    dt = g.cfl()
    assert f.cfl_limit() == dt
    with pytest.raises(RuntimeError) as eg:
        g.step(dt)
    with pytest.raises(RuntimeError) as ef:
        f.step_unchecked(dt)
    assert "cannot advance time" in str(eg.value)
    assert str(ef.value) == str(eg.value)


@pytest.mark.parametrize("name", ["orszag_tang", "rotor", "blast", "brio_wu", "alfven_wave"])
@pytest.mark.parametrize("recon", ["mp5", "mp7"])
def test_reference_seed_on_seam_matches_cpu_seed(seam, ref, name, recon):
    """The reference's own build_initial_state (initial_conditions.cpp:166-213)
    seeding through launch_mhd_seed_initial_state, here this project's
    kernels, against the same call in the reference's CPU build.  Bit for bit
    for brio_wu and blast; where CUDA's sin, cos or hypot differ from the C
    library's in the last bit (a few Orszag-Tang and Alfven-wave cells, two
    rotor taper cells), every component agrees within 8 ulp of its largest
    magnitude."""
    import copy
    import deck_cases as D
    from quasar_b200 import deck as Q
    d = Q.parse(copy.deepcopy(D.decks(recon=recon)[name]))
    dm = d.domain
    args = (Q._KIND[d.initial.type], dm.nx, dm.ny, dm.lx_m, dm.ly_m, dm.origin_x_m,
            dm.origin_y_m, Q.nghost(recon), d.numerics.gamma, {"mp5": 5, "mp7": 7}[recon])
    got = seam.initial_state(*args, **D.ref_params(d))
    want = ref.initial_state(*args, **D.ref_params(d))
    eps = np.finfo(np.float64).eps
    for c, comp in enumerate(Q.STATE_COMPONENTS):
        a, b = got[c], want[c]
        assert np.all(np.isfinite(a)), (name, comp)
        if name in ("brio_wu", "blast"):
            assert np.array_equal(a, b), (name, comp)
        else:
            scale = max(float(np.abs(b).max()), 1e-300)
            assert float(np.abs(a - b).max()) <= 8 * eps * scale, (
                name, comp, float(np.abs(a - b).max()), scale)
