"""Initial-state families without a reference generator (quasar_b200.ics):
exact discrete solenoidality of the oblique fields, the wave eigenvectors,
the seeded batch description, and that the reference's own CPU solver
(oracle/_ref) accepts and steps every family."""
import math

import numpy as np
import pytest

import mhd_cases as M
from quasar_b200 import ics


def discrete_div(bx, by, dx, dy):
    """The solver's per-cell divergence, (bx_h - bx_l)/dx + (by_h - by_l)/dy."""
    return (bx[:-1, 1:] - bx[:-1, :-1]) / dx + (by[1:, :-1] - by[:-1, :-1]) / dy


@pytest.mark.parametrize("angle", [0.0, 0.37, 0.79, 1.21, 1.57])
def test_oblique_fields_are_exactly_solenoidal(angle):
    for order in (5, 7):
        nx, ny = 53, 38
        for arrays, lx, ly, _ in (ics.brio_wu_rotated(nx, ny, order=order, angle=angle),
                                  ics.linear_wave(nx, ny, order=order, angle=angle),
                                  ics.linear_wave(nx, ny, order=order, angle=angle,
                                                  kind="alfven")):
            d = discrete_div(arrays[5], arrays[6], lx / nx, ly / ny)
            assert np.all(d == 0.0)


def test_oblique_direction_is_commensurate():
    arrays, lx, ly, th = ics.brio_wu_rotated(64, 48, order=5, angle=0.9)
    assert abs(th - 0.9) < 0.2
    # periodic: the interior pattern repeats across the box
    ng = 3
    rho = arrays[0][ng:-ng, ng:-ng]
    assert set(np.unique(rho)) == {0.125, 1.0}


def test_wave_eigenvectors():
    r, w = ics._wave_eigenvector("fast", 1.0, 0.6, 1.0, math.sqrt(2.0), 0.5, 5.0 / 3.0)
    a2, b2, bn2 = 1.0, 1.0 + 2.0 + 0.25, 1.0
    cf = math.sqrt(0.5 * (a2 + b2 + math.sqrt((a2 + b2) ** 2 - 4 * a2 * bn2)))
    assert abs(w - cf) < 1e-12
    r, w = ics._wave_eigenvector("alfven", 1.0, 0.6, 1.0, math.sqrt(2.0), 0.5, 5.0 / 3.0)
    assert abs(w - 1.0) < 1e-12
    assert abs(r[0]) < 1e-12 and abs(r[4]) < 1e-12  # incompressible


def test_batch_description_is_seeded_and_deterministic():
    a = ics.batch_instances()
    b = ics.batch_instances()
    assert len(a) == 256
    assert [(x["family"], x["nx"], x["ny"]) for x in a] == [(x["family"], x["nx"], x["ny"]) for x in b]
    fams = {x["family"] for x in a}
    assert fams == {"orszag_tang", "brio_wu", "fast_wave", "alfven_wave"}
    assert all(64 <= x["nx"] <= 512 and 64 <= x["ny"] <= 512 for x in a)


def test_reference_solver_steps_every_family(ref):
    for inst in ics.batch_instances(count=8, seed=5, lo=24, hi=40):
        bc = M.PERIODIC if inst["bc"] == 0 else M.OUTFLOW
        s = ref.solver(inst["nx"], inst["ny"], 5, gamma=inst["gamma"], bc=bc,
                       lx=inst["lx"], ly=inst["ly"])
        s.seed(inst["arrays"]())
        for _ in range(2):
            s.step(s.cfl())
