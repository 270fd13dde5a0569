"""Batched instances (include/quasar_mhd_batch.h) on the GPU, through the C ABI.

A batched step runs the same device bodies as the single-instance step over
tables of every instance's arguments; inlined into different kernels they
may contract multiply-adds differently, so each instance must end within
rounding of where it ends when stepped alone: every component within
BATCH_TOL of the state's largest magnitude (a per-group relative measure
would divide by the 1e-6 momentum of a linear wave).  The autotuner only
changes launch grids.
The oblique families of quasar_b200.ics (no reference generator) are pinned
against the oracle restatement step by step like the reference's own ICs."""
import numpy as np
import pytest

import mhd_cases as M
from quasar_b200 import ics, mhd

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10
BATCH_TOL = 1e-12


def config(inst, order):
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(inst["nx"], inst["ny"], inst["lx"], inst["ly"])
    cfg.reconstruction = "mp7" if order == 7 else "mp5"
    cfg.gamma = inst["gamma"]
    bc = "periodic" if inst["bc"] == 0 else "outflow"
    cfg.boundary = mhd.MhdBoundarySpec([bc] * 4, [bc] * 4)
    return cfg


def mixed_instances(order, count=6, seed=11):
    out = ics.batch_instances(count=count, seed=seed, lo=24, hi=72, order=order)
    n = max(24, 40)
    out.append(dict(family="rotor", nx=n, ny=n + 8, lx=1.0, ly=1.0, gamma=5.0 / 3.0, bc=1,
                    arrays=lambda: ics.rotor(n, order=order, ny=n + 8)))
    return out


def rounding_gap(a, b):
    """max over components of max|a - b|, relative to the largest |b|."""
    scale = max(float(np.max(np.abs(v))) for v in b)
    return max(float(np.max(np.abs(u - v))) for u, v in zip(a, b)) / scale


def read_all(s, inst, order):
    ng = ics.nghost(order)
    shape = (inst["ny"] + 2 * ng, inst["nx"] + 2 * ng)
    return [s.state_component_to_host(c).reshape(shape) for c in ics.COMPONENTS]


@pytest.mark.parametrize("order", [5, 7])
def test_batch_equals_each_instance_alone(order):
    insts = mixed_instances(order)
    b = mhd.MhdBatch2D([config(x, order) for x in insts])
    alone = [mhd.MhdSolver2D(config(x, order)) for x in insts]
    for i, x in enumerate(insts):
        arrays = x["arrays"]()
        for name, a in zip(ics.COMPONENTS, arrays):
            b.instance(i).seed_state(name, a)
            alone[i].seed_state(name, a)
    assert b.zones() == sum(x["nx"] * x["ny"] for x in insts)
    done = b.advance(5)
    assert done == [5] * len(insts)
    for i, x in enumerate(insts):
        t, k = alone[i].advance_auto(0.0, 1e30, 5)
        assert k == 5
        err = rounding_gap(read_all(b.instance(i), x, order), read_all(alone[i], x, order))
        assert err <= BATCH_TOL, (x["family"], i, err)
        assert b.instance(i).divergence_b_max() <= 1e-12


def test_autotuned_batch_still_equals_instances():
    order = 5
    insts = mixed_instances(order, count=5, seed=12)
    b = mhd.MhdBatch2D([config(x, order) for x in insts])
    alone = [mhd.MhdSolver2D(config(x, order)) for x in insts]
    for i, x in enumerate(insts):
        arrays = x["arrays"]()
        for name, a in zip(ics.COMPONENTS, arrays):
            b.instance(i).seed_state(name, a)
            alone[i].seed_state(name, a)
    ctas, trials = b.autotune()
    assert len(ctas) == mhd.MhdBatch2D.PHASES and trials >= 2
    done = b.advance(3)
    for i, x in enumerate(insts):
        _, k = alone[i].advance_auto(0.0, 1e30, trials + done[i])
        err = rounding_gap(read_all(b.instance(i), x, order), read_all(alone[i], x, order))
        assert err <= BATCH_TOL, (x["family"], i, err)
    ms, zu = b.time_steps(2)
    assert ms > 0 and zu == 2 * b.zones()


def test_profiled_batch_step_is_a_batched_step():
    """qmhd_batch_profile_step: one step of every instance (the same state as
    stepping each alone) with a non-negative device time per phase."""
    order = 7
    insts = mixed_instances(order, count=3, seed=14)
    b = mhd.MhdBatch2D([config(x, order) for x in insts])
    alone = [mhd.MhdSolver2D(config(x, order)) for x in insts]
    for i, x in enumerate(insts):
        for name, a in zip(ics.COMPONENTS, x["arrays"]()):
            b.instance(i).seed_state(name, a)
            alone[i].seed_state(name, a)
    ph = b.profile_step()
    assert len(ph) == mhd.MhdBatch2D.PHASES + 1
    assert all(np.isfinite(v) and v >= 0.0 for v in ph.values()) and sum(ph.values()) > 0.0
    for i, x in enumerate(insts):
        _, k = alone[i].advance_auto(0.0, 1e30, 1)
        assert k == 1
        err = rounding_gap(read_all(b.instance(i), x, order), read_all(alone[i], x, order))
        assert err <= BATCH_TOL, (x["family"], i, err)


def test_batch_rejects_mixed_orders():
    insts = mixed_instances(5, count=2)
    with pytest.raises(ValueError):
        mhd.MhdBatch2D([config(insts[0], 5), config(insts[1], 7)])


@pytest.mark.parametrize("family", ["brio_wu", "fast_wave", "alfven_wave"])
def test_oblique_families_match_oracle(oracle, family):
    order, nx, ny = 5, 40, 28
    if family == "brio_wu":
        arrays, lx, ly, _ = ics.brio_wu_rotated(nx, ny, order=order, angle=0.6)
        gamma = 2.0
    else:
        arrays, lx, ly, _ = ics.linear_wave(nx, ny, order=order, angle=1.0,
                                            kind=family.split("_")[0])
        gamma = 5.0 / 3.0
    inst = dict(nx=nx, ny=ny, lx=lx, ly=ly, gamma=gamma, bc=0)
    g = mhd.MhdSolver2D(config(inst, order))
    o = oracle.solver(nx, ny, order, gamma=gamma, bc=M.PERIODIC, lx=lx, ly=ly)
    for name, a in zip(ics.COMPONENTS, arrays):
        g.seed_state(name, a)
    o.seed(arrays)
    ng = ics.nghost(order)
    for k in range(4):
        dt, dto = g.cfl_limit(), o.cfl()
        assert abs(dt - dto) <= 1e-12 * dto, (k, dt, dto)
        g.step_unchecked(dto)
        o.step(dto)
        err = M.state_rel_l1(read_all(g, inst, order), o.read(), ng, nx, ny)
        assert err <= STEP_TOL, (k, err)
    assert g.divergence_b_max() <= 1e-12


DIVB_NOISE = 2.0  # spread of two round-off random walks of the same statistics


def _seeded_pair(order, count, seed):
    insts = mixed_instances(order, count=count, seed=seed)
    b = mhd.MhdBatch2D([config(x, order) for x in insts])
    c = mhd.MhdBatch2D([config(x, order) for x in insts])
    for i, x in enumerate(insts):
        arrays = x["arrays"]()
        for name, a in zip(ics.COMPONENTS, arrays):
            b.instance(i).seed_state(name, a)
            c.instance(i).seed_state(name, a)
    return insts, b, c


def test_batched_learned_with_every_cell_flagged_is_the_batched_step():
    from quasar_b200.indicator import TroubledCellIndicator, attach_batch
    order = 5
    insts, b, c = _seeded_pair(order, 5, 21)
    ind = TroubledCellIndicator(seed=3)
    attach_batch(ind, c, -1e30)
    assert b.advance(4) == [4] * len(insts)
    assert c.advance(4) == [4] * len(insts)
    for i, x in enumerate(insts):
        err = rounding_gap(read_all(c.instance(i), x, order), read_all(b.instance(i), x, order))
        assert err <= BATCH_TOL, (x["family"], i, err)


def test_batched_learned_with_shipped_indicator_stays_close():
    from quasar_b200 import train_indicator
    from quasar_b200.indicator import attach_batch
    order = 5
    insts, b, c = _seeded_pair(order, 6, 22)
    ind, thr = train_indicator.load(order=order)
    attach_batch(ind, c, thr)
    b.advance(20)
    c.advance(20)
    ng = ics.nghost(order)
    for i, x in enumerate(insts):
        rb = read_all(b.instance(i), x, order)[0][ng:-ng, ng:-ng]
        rc = read_all(c.instance(i), x, order)[0][ng:-ng, ng:-ng]
        l1 = np.sum(np.abs(rc - rb)) / np.sum(np.abs(rb))
        assert l1 <= 1e-4, (x["family"], i, l1)
        # solenoidality in the reference's relative measure and bound
        # (tests/python/test_examples.py:1985-2003), and at the plain run's
        # own round-off level: CT keeps div B exact in exact arithmetic for
        # any EMF, so both runs carry a random walk of the same rounding
        # statistics (DIVB_NOISE allows for its spread)
        rel_l, rel_p = c.instance(i).divergence_b_relative(), b.instance(i).divergence_b_relative()
        assert rel_l < 1e-11 and rel_l <= DIVB_NOISE * max(rel_p, 1e-15), (x["family"], i, rel_l, rel_p)
