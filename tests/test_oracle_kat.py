"""The oracle restatement against the known answers of the reference's own
unit tests (read as text; the numbers are the reference's)."""
import numpy as np

import mhd_cases as M


def conserved(rho, vx, vy, vz, p, bx, by, bz, gamma):
    # tests/unit/numerics/test_hlld_riemann.cpp:50-64
    e_int = p / ((gamma - 1.0) * rho)
    return np.array([rho, rho * vx, rho * vy, rho * vz,
                     rho * e_int + 0.5 * rho * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz),
                     bx, by, bz])


def test_hlld_right_double_star_energy_golden(oracle):
    # test_hlld_riemann.cpp:357-376: energy flux -2.0871013232600024 +- 2e-13
    g = 5.0 / 3.0
    L = conserved(0.5, 0.2, 0.8, -0.3, 0.7, 0.9, 0.4, 0.5, g)
    R = conserved(1.4, -0.5, -0.2, 0.9, 1.2, 0.9, -0.7, -0.1, g)
    f = oracle.hlld_flux_x(L, R, g)
    assert abs(f[4] - (-2.0871013232600024)) <= 2e-13
    assert abs(f[4] - (-1.9282917918373412)) > 0.1


def test_hlld_consistency(oracle):
    g = 5.0 / 3.0
    U = conserved(1.1, 0.3, -0.2, 0.1, 0.9, 0.7, -0.4, 0.25, g)
    f = oracle.hlld_flux_x(U, U, g)
    vx, vy, vz = U[1] / U[0], U[2] / U[0], U[3] / U[0]
    bx, by, bz = U[5:8]
    p = (g - 1) * (U[4] - 0.5 * U[0] * (vx * vx + vy * vy + vz * vz) - 0.5 * (bx * bx + by * by + bz * bz))
    pt = p + 0.5 * (bx * bx + by * by + bz * bz)
    exact = [U[1], U[1] * vx + pt - bx * bx, U[1] * vy - bx * by, U[1] * vz - bx * bz,
             (U[4] + pt) * vx - bx * (vx * bx + vy * by + vz * bz), 0.0, by * vx - bx * vy, bz * vx - bx * vz]
    assert np.allclose(f, exact, rtol=1e-14, atol=1e-14)


def test_mp_limiter_kats(oracle):
    # tests/unit/numerics/test_mp_limiter.cpp:36-128
    assert abs(oracle.mp([3.5] * 5) - 3.5) <= 1e-12
    assert abs(oracle.mp([3.5] * 7) - 3.5) <= 1e-12
    assert abs(oracle.mp([0, 0, 1, 1, 1]) - 1.0) <= 1e-9
    assert abs(oracle.mp([0, 0, 0, 0, 1]) - 0.0) <= 1e-9
    assert abs(oracle.mp([0, 0, 0, 1, 1, 1, 1]) - 1.0) <= 1e-9
    a = 1e-100
    lim = oracle.mp([0, 0, a, a, a])
    assert lim <= a and lim >= 0 and abs(lim / a - 1.0) <= 1e-12
    v = [1.0] * 6 + [0.0] * 6
    for i in range(2, 10):
        w = v[i - 2:i + 3]
        lim = oracle.mp(w)
        assert min(w) - 1e-12 <= lim <= max(w) + 1e-12


def test_oracle_matches_reference_kernels(oracle, ref):
    g = 5.0 / 3.0
    rng = np.random.default_rng(3)
    for _ in range(50):
        L = conserved(*rng.uniform(0.2, 2.0, 1), *rng.normal(0, 1, 3), *rng.uniform(0.1, 2.0, 1), *rng.normal(0, 1, 3), g)
        R = conserved(*rng.uniform(0.2, 2.0, 1), *rng.normal(0, 1, 3), *rng.uniform(0.1, 2.0, 1), *rng.normal(0, 1, 3), g)
        R[5] = L[5]
        a, b = oracle.hlld_flux_x(L, R, g), ref.hlld_flux_x(L, R, g)
        assert np.allclose(a, b, rtol=1e-13, atol=1e-13)
        w = rng.normal(0, 1, 7)
        assert abs(oracle.mp(w) - ref.mp(w)) <= 1e-13
        assert abs(oracle.mp(w[:5]) - ref.mp(w[:5])) <= 1e-13


def test_mlp_oracle_gradient_matches_finite_differences(monkeypatch):
    """The indicator network's CPU restatement: analytic gradient against
    central differences (BF16 operand rounding switched off)."""
    import os
    import sys
    import numpy as np
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import mlp_oracle as O
    monkeypatch.setattr(O, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    rng = np.random.default_rng(0)
    p = rng.standard_normal(O.NPARAM) * 0.1
    X = rng.standard_normal((40, O.FEAT))
    y = (rng.random(40) < 0.3).astype(float)
    _, g = O.loss_and_grads(p, X, y, pos_weight=3.0)
    idx = np.concatenate([rng.integers(0, O.NPARAM, 40), [O.NPARAM - 1]])
    h = 1e-6
    for i in idx:
        e = np.zeros(O.NPARAM)
        e[i] = h
        fd = (O.loss_and_grads(p + e, X, y, 3.0)[0] - O.loss_and_grads(p - e, X, y, 3.0)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
