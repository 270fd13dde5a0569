"""Pin the oracle restatement against the reference's own solver (built for
the CPU in oracle/_ref) and against the committed reference fixtures."""
import os

import numpy as np
import pytest

import mhd_cases as M

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"ot": M.orszag_tang, "rotor": M.rotor, "blast": M.blast}
SHORT = ["ot32_mp5", "ot32_mp7", "rotor32_mp7", "blast32_mp7", "rotor48_mp5", "ot24_muscl"]


def load_fixture(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", SHORT)
def test_oracle_matches_reference_fixture(oracle, name):
    fx = load_fixture(name)
    n, order, case = int(fx["n"]), int(fx["order"]), str(fx["case"])
    bc = tuple(int(b) for b in fx["bc"])
    s = oracle.solver(n, n, order, bc=bc)
    s.seed(CASES[case](n, order=order))
    for k, dt_ref in enumerate(fx["dts"]):
        dt = s.cfl()
        # dt is a max-reduction of comparison-only operations: bit-exact but
        # for the rounding of the per-face rates
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref, (k, dt, dt_ref)
        s.step(dt_ref)
    got = s.read()
    want = [fx[c] for c in M.COMPONENTS]
    assert M.state_rel_l1(got, want, s.ng, n, n) <= 1e-13


@pytest.mark.parametrize("name", ["rotor512_mp7", "blast512_mp7"])
def test_oracle_matches_reference_at_benchmark_workloads_512(oracle, name):
    """The benchmark's rotor and blast MP7 workloads at 512^2: two steps of
    the oracle against the reference's summary fixtures."""
    fx = load_fixture(name)
    n, order, case = int(fx["n"]), int(fx["order"]), str(fx["case"])
    s = oracle.solver(n, n, order, bc=tuple(int(b) for b in fx["bc"]))
    s.seed(CASES[case](n, order=order))
    for k, dt_ref in enumerate(fx["dts"]):
        dt = s.cfl()
        assert abs(dt - dt_ref) <= 1e-13 * dt_ref, (k, dt, dt_ref)
        s.step(dt_ref)
    assert M.summary_rel(s.read(), fx, n, order) <= 1e-13


def test_oracle_residual_matches_reference(oracle, ref):
    n, order = 24, 7
    ic = M.rotor(n, order=order)
    a = oracle.solver(n, n, order, bc=M.OUTFLOW).residual(ic)
    b = ref.solver(n, n, order, bc=M.OUTFLOW).residual(ic)
    for c in range(8):
        scale = max(np.abs(b["dudt"][c]).max(), 1.0)
        assert np.abs(a["dudt"][c] - b["dudt"][c]).max() <= 1e-12 * scale


def test_oracle_positivity_retry_matches_reference(oracle, ref):
    """A strong blast at 16^2 with an aggressive dt enters the positivity
    controller in both (mhd_solver.cpp:965-1143)."""
    n, order = 16, 5
    ic = M.blast(n, order=order)
    ic[4] = np.where(ic[4] > 100, ic[4] * 1e3, ic[4])
    so, sr = oracle.solver(n, n, order, bc=M.OUTFLOW), ref.solver(n, n, order, bc=M.OUTFLOW)
    so.seed(ic)
    sr.seed(ic)
    dt = 3.0 * sr.cfl()
    so.step(dt)
    sr.step(dt)
    assert so.substeps() == sr.substeps()
    assert M.state_rel_l1(so.read(), sr.read(), so.ng, n, n) <= 1e-12


def test_oracle_count_is_positive(oracle):
    s = oracle.solver(16, 16, 5, counting=True)
    s.seed(M.orszag_tang(16, order=5))
    as_written, alg, cfl = oracle.count_flops(s, 1)
    assert as_written > alg > 10000 and cfl > 0
