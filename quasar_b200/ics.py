"""Benchmark initial states as padded host arrays (reference storage layout).

Profiles follow the reference's analytic initial-condition generators
(src/backend/hip/mhd/mhd_initial_conditions.hip:116-188): primitives at cell
centres, magnetic field sampled on its own faces, conserved energy
p/(gamma-1) + rho|v|^2/2 + |B|^2/2.  Arrays are (ny+2g, nx+2g) C-order, so the
flat index is (i+g) + (nx+2g)(j+g); components rho, mx, my, mz, energy,
bx_face, by_face, bz_cell.
"""
from __future__ import annotations

import math

import numpy as np

COMPONENTS = ("rho", "mx", "my", "mz", "energy", "bx_face", "by_face", "bz_cell")


def nghost(order: int) -> int:
    return 4 if order == 7 else 3 if order == 5 else 2


def _centres(n, ng, length=1.0, origin=0.0):
    return (np.arange(-ng, n + ng, dtype=np.float64) + 0.5) * (length / n) + origin


def _assemble(rho, vx, vy, vz, p, bx, by, bz, gamma):
    kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    mag = 0.5 * (bx * bx + by * by + bz * bz)
    energy = p / (gamma - 1.0) + kin + mag
    return [np.ascontiguousarray(a, dtype=np.float64) for a in
            (rho, rho * vx, rho * vy, rho * vz, energy, bx, by, bz)]


def orszag_tang(n, order=5, gamma=5.0 / 3.0, amplitude=1.0, ny=None):
    """rho=25a/(36 pi), p=5a/(12 pi), v=(-sin 2 pi y, sin 2 pi x),
    face B = sqrt(a)/sqrt(4 pi) (-sin 2 pi y, sin 4 pi x) on [0,1]^2."""
    ny = n if ny is None else ny
    ng = nghost(order)
    X, Y = np.meshgrid(_centres(n, ng), _centres(ny, ng), indexing="xy")
    pi = math.pi
    rho = np.full_like(X, amplitude * 25.0 / (36.0 * pi))
    p = np.full_like(X, amplitude * 5.0 / (12.0 * pi))
    b0 = math.sqrt(amplitude) / math.sqrt(4.0 * pi)
    z = np.zeros_like(X)
    return _assemble(rho, -np.sin(2 * pi * Y), np.sin(2 * pi * X), z, p,
                     -b0 * np.sin(2 * pi * Y), b0 * np.sin(4 * pi * X), z, gamma)


def rotor(n, order=7, gamma=5.0 / 3.0):
    """rho=10 for r<0.1, linear taper to 1 at r=0.115, rigid rotation u0=2 at
    r0=0.1 tapering to rest at r1, p=1, Bx=5/sqrt(4 pi) (mhd_initial_conditions.hip:159-188)."""
    ng = nghost(order)
    X, Y = np.meshgrid(_centres(n, ng), _centres(n, ng), indexing="xy")
    rx, ry = X - 0.5, Y - 0.5
    r = np.hypot(rx, ry)
    r0, r1, u0 = 0.1, 0.115, 2.0
    f = np.clip((r1 - r) / (r1 - r0), 0.0, 1.0)
    f = np.where(r <= r0, 1.0, np.where(r >= r1, 0.0, f))
    with np.errstate(divide="ignore", invalid="ignore"):
        sf = np.where(r <= r0, u0 / r0, np.where(r < r1, f * u0 / np.maximum(r, 1e-300), 0.0))
    z = np.zeros_like(X)
    return _assemble(1.0 + f * 9.0, -sf * ry, sf * rx, z, np.ones_like(X),
                     np.full_like(X, 5.0 / math.sqrt(4.0 * math.pi)), z, z, gamma)


def blast(n, order=7, gamma=5.0 / 3.0):
    """p=100 for r<0.1 else 0.1, rho=1, Bx=By=10/sqrt(8 pi) (mhd_initial_conditions.hip:145-157)."""
    ng = nghost(order)
    X, Y = np.meshgrid(_centres(n, ng), _centres(n, ng), indexing="xy")
    r = np.hypot(X - 0.5, Y - 0.5)
    b = 10.0 / math.sqrt(8.0 * math.pi)
    z = np.zeros_like(X)
    return _assemble(np.ones_like(X), z, z, z, np.where(r < 0.1, 100.0, 0.1),
                     np.full_like(X, b), np.full_like(X, b), z, gamma)


GENERATORS = {"orszag_tang": orszag_tang, "rotor": rotor, "blast": blast}
