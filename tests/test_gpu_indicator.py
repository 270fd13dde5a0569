"""Tensor-core troubled-cell indicator against its numpy restatement
(oracle/mlp_oracle.py), through the C ABI."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


def random_rows(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((n, O.FEAT)) * 0.7).astype(np.float32)


@pytest.mark.parametrize("rows", [1, 127, 128, 1000, 40000])
def test_forward_matches_oracle(rows):
    from quasar_b200.indicator import TroubledCellIndicator
    ind = TroubledCellIndicator(seed=3)
    p = ind.params()
    rng = np.random.default_rng(4)
    p[O.HID * O.FEAT:O.HID * O.FEAT + O.HID] = rng.standard_normal(O.HID) * 0.1  # b1
    ind.set_params(p)
    x = random_rows(rows, rows)
    got = ind.forward(x)
    want, _ = O.forward(p, x)
    scale = np.max(np.abs(want)) + 1e-30
    assert np.max(np.abs(got - want)) <= 2e-3 * scale, np.max(np.abs(got - want)) / scale


def test_gradient_matches_oracle():
    from quasar_b200.indicator import TroubledCellIndicator
    ind = TroubledCellIndicator(seed=5)
    p = ind.params()
    rng = np.random.default_rng(6)
    p += (rng.standard_normal(p.shape) * 0.02).astype(np.float32)
    ind.set_params(p)
    x = random_rows(1000, 7)
    y = (rng.random(1000) < 0.3).astype(np.uint8)
    loss, g = ind.gradient(x, y, pos_weight=3.0)
    lo, go = O.loss_and_grads(p.astype(np.float64), x, y, pos_weight=3.0)
    assert abs(loss - lo) <= 1e-4 * abs(lo)
    o = 0
    for name, size in (("w1", O.HID * O.FEAT), ("b1", O.HID), ("w2", O.HID * O.HID),
                       ("b2", O.HID), ("w3", O.HID), ("b3", 1)):
        a, b = g[o:o + size], go[o:o + size]
        rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30)
        assert rel <= 2e-2, (name, rel)
        o += size


def _ot_solver(n, order=5):
    from quasar_b200 import ics, mhd
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(n, n, 1.0, 1.0)
    cfg.reconstruction = "mp5" if order == 5 else "mp7"
    s = mhd.MhdSolver2D(cfg)
    for name, a in zip(ics.COMPONENTS, ics.orszag_tang(n, order=order)):
        s.seed_state(name, a)
    return s


def _state(s):
    from quasar_b200 import ics
    return [s.state_component_to_host(c) for c in ics.COMPONENTS]


@pytest.mark.parametrize("order", [5, 7])
def test_learned_mode_with_every_cell_flagged_is_the_plain_step(order):
    from quasar_b200.indicator import TroubledCellIndicator, learned_face_counts
    n = 48
    a, b = _ot_solver(n, order), _ot_solver(n, order)
    ind = TroubledCellIndicator(seed=1)
    ind.attach(b, -1e30)
    for _ in range(3):
        a.step_unchecked(a.cfl_limit())
        b.step_unchecked(b.cfl_limit())
    ua, ub = _state(a), _state(b)
    scale = max(np.max(np.abs(v)) for v in ua)
    gap = max(np.max(np.abs(x - y)) for x, y in zip(ub, ua)) / scale
    assert gap <= 1e-12, gap
    ng = 3 if order == 5 else 4
    fx, fy = learned_face_counts(b)
    assert fx == (n + 1) * (n + 2 * ng) and fy == (n + 1) * (n + 2 * ng)


def test_collect_train_and_learned_steps():
    from quasar_b200.indicator import TroubledCellIndicator, learned_face_counts
    n = 64
    s = _ot_solver(n)
    ind = TroubledCellIndicator(seed=2)
    for k in range(40):
        s.step_unchecked(s.cfl_limit())
        if k % 4 == 3:
            ind.collect(s)
    assert ind.rows() == 10 * n * n
    l0 = ind.train(epochs=1, tiles_per_step=16, lr=1e-3, pos_weight=4.0, holdout=10)
    l1 = ind.train(epochs=6, tiles_per_step=16, lr=1e-3, pos_weight=4.0, holdout=10)
    assert np.isfinite(l1) and l1 < l0
    thr = ind.threshold_for_recall(0.99, holdout=10)
    ev = ind.evaluate(thr, holdout=10)
    assert ev["recall"] >= 0.99 and ev["positives"] > 0
    # learned steps against plain ones from the same state
    a, b = _ot_solver(n), _ot_solver(n)
    for _ in range(30):
        a.step_unchecked(a.cfl_limit())
        b.step_unchecked(b.cfl_limit())
    ind.attach(b, thr)
    for _ in range(10):
        a.step_unchecked(a.cfl_limit())
        b.step_unchecked(b.cfl_limit())
    fx, fy = learned_face_counts(b)
    assert fx < (n + 1) * (n + 6)
    ra, rb = _state(a)[0], _state(b)[0]
    l1 = np.sum(np.abs(ra - rb)) / np.sum(np.abs(ra))
    assert l1 <= 1e-3, l1
    assert b.divergence_b_max() <= 1e-12


def test_inference_report_on_developed_orszag_tang():
    """The shipped MP5 indicator at inference on Orszag-Tang 512^2 after the
    shocks have formed (t = 0.3): the learned step stays within 1e-4 of the
    plain one in density L1 and its flags catch most of the plain limiter's
    activations while keeping most faces on the cheap path."""
    from quasar_b200 import train_indicator
    r = train_indicator.inference_report(512, 5, t_develop=0.3, steps=60)
    assert r["limiter_positive"] > 1000
    assert r["rho_l1_vs_plain"] <= 1e-4
    assert r["limiter_recall"] >= 0.8
    assert r["cells_flagged"] < 0.35 and r["full_path_face_fraction"] < 0.35
    # solenoidality in the reference's relative measure and bound
    # (tests/python/test_examples.py:1985-2003), at the plain run's own
    # round-off level (both are random walks of the same rounding statistics)
    assert r["div_b_rel"] < 1e-11, r
    assert r["div_b_rel"] <= 2.0 * max(r["div_b_rel_plain"], 1e-15), r


def _tube(n, order, axis):
    """A Brio-Wu-like tube varying along one axis only (outflow): the normal
    field uniform, the tangential field and the gas jumping at the middle."""
    from quasar_b200 import ics, mhd
    ng = ics.nghost(order)
    X, Y = np.meshgrid(ics._centres(n, ng, 1.0, 0.0), ics._centres(n, ng, 1.0, 0.0), indexing="xy")
    s = X if axis == 0 else Y
    left = s < 0.5
    rho, p = np.where(left, 1.0, 0.125), np.where(left, 1.0, 0.1)
    bt = np.where(left, 1.0, -1.0)
    zero = np.zeros_like(X)
    bx, by = (zero + 0.75, bt) if axis == 0 else (bt, zero + 0.75)
    comps = ics._assemble(rho, zero, zero, zero, p, bx, by, zero, 2.0)
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(n, n, 1.0, 1.0)
    cfg.reconstruction = "mp5" if order == 5 else "mp7"
    cfg.gamma = 2.0
    cfg.boundary = mhd.MhdBoundarySpec(["outflow"] * 4, ["outflow"] * 4)
    sv = mhd.MhdSolver2D(cfg)
    for name, a in zip(ics.COMPONENTS, comps):
        sv.seed_state(name, a)
    return sv


@pytest.mark.parametrize("order", [5, 7])
def test_labels_come_from_both_face_directions(order):
    """Limiter labels of a tube along x and of the same tube along y: only the
    faces normal to the tube see its jump, so the labels of one come from x
    faces and of the other from y faces alone; by symmetry their counts agree,
    and both orders collect."""
    from quasar_b200.indicator import TroubledCellIndicator
    counts = []
    for axis in (0, 1):
        s = _tube(64, order, axis)
        for _ in range(4):
            s.step_unchecked(s.cfl_limit())
        ind = TroubledCellIndicator(seed=0)
        ind.collect(s, 1e-4)
        counts.append(ind.evaluate(0.0, holdout=0)["positives"])
    assert counts[0] > 0 and counts[0] == counts[1], counts


def test_trained_indicator_beats_untrained_and_heuristic():
    """What training buys, on a developed Orszag-Tang 512^2 MP5 state: at the
    same 95% recall of the plain limiter's activations, the shipped network
    flags fewer cells than the untrained network and than a density/pressure
    jump threshold, and the learned step at its shipped threshold stays within
    1e-4 of the plain step in density L1."""
    from quasar_b200 import train_indicator
    r = train_indicator.gain_report(512, 5, t_develop=0.3, steps=60)
    assert r["positives"] > 1000, r
    assert r["trained"]["recall"] >= 0.95 and r["untrained"]["recall"] >= 0.95, r
    assert r["trained"]["flagged"] < r["heuristic"]["flagged"], r
    assert r["trained"]["flagged"] < r["untrained"]["flagged"], r
    assert r["rho_l1_vs_plain"] <= 1e-4, r
    assert 0.0 < r["literal_label"]["positive_fraction"] <= 1.0, r
