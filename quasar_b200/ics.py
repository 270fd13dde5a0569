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


def rotor(n, order=7, gamma=5.0 / 3.0, ny=None, r0=0.1, bx=5.0 / math.sqrt(4.0 * math.pi)):
    """rho=10 for r<r0, linear taper to 1 at r1 = 1.15 r0, rigid rotation
    u0=2 at r0 tapering to rest at r1, p=1, Bx=5/sqrt(4 pi)
    (mhd_initial_conditions.hip:159-188)."""
    ng = nghost(order)
    ny = n if ny is None else ny
    X, Y = np.meshgrid(_centres(n, ng), _centres(ny, ng), indexing="xy")
    rx, ry = X - 0.5, Y - 0.5
    r = np.hypot(rx, ry)
    r1, u0 = 0.115 * (r0 / 0.1), 2.0  # 0.115 exactly at the default radius
    f = np.clip((r1 - r) / (r1 - r0), 0.0, 1.0)
    f = np.where(r <= r0, 1.0, np.where(r >= r1, 0.0, f))
    with np.errstate(divide="ignore", invalid="ignore"):
        sf = np.where(r <= r0, u0 / r0, np.where(r < r1, f * u0 / np.maximum(r, 1e-300), 0.0))
    z = np.zeros_like(X)
    return _assemble(1.0 + f * 9.0, -sf * ry, sf * rx, z, np.ones_like(X),
                     np.full_like(X, bx), z, z, gamma)


def blast(n, order=7, gamma=5.0 / 3.0, ny=None, radius=0.1, p_in=100.0, p_out=0.1,
          b=10.0 / math.sqrt(8.0 * math.pi)):
    """p=100 for r<0.1 else 0.1, rho=1, Bx=By=10/sqrt(8 pi) (mhd_initial_conditions.hip:145-157)."""
    ng = nghost(order)
    ny = n if ny is None else ny
    X, Y = np.meshgrid(_centres(n, ng), _centres(ny, ng), indexing="xy")
    r = np.hypot(X - 0.5, Y - 0.5)
    z = np.zeros_like(X)
    return _assemble(np.ones_like(X), z, z, z, np.where(r < radius, p_in, p_out),
                     np.full_like(X, b), np.full_like(X, b), z, gamma)


# ---- families without a reference generator --------------------------------
# The reference's Brio-Wu tube is x-aligned and its Alfven wave x-propagating
# (mhd_initial_conditions.hip:67-114).  Oblique versions take the in-plane
# field from a corner vector potential A_z (B = curl A, the stencil of
# launch_mhd_curl_corner_potential, physics/mhd/kernels.hpp:725-728).  A
# seeded field must be discretely divergence-free to the bit (mhd_solver.cpp
# 1196-1222 accepts round-off only where both derivatives cancel), so the
# field is built on an exact lattice: cells of side h = 2^-9, the periodic
# part of A rounded to multiples of q = h 2^-35 on the periodic corner
# lattice and the uniform part rounded to multiples of 2^-35.  Every face
# value, face difference and divided difference is then exact in binary64
# and the discrete divergence is exactly zero.

_F2C = {6: ([11, -93, 802, 802, -93, 11], 1440.0),
        8: ([-191, 1879, -9531, 68323, 68323, -9531, 1879, -191], 120960.0),
        4: ([-1, 13, 13, -1], 24.0)}


def _collocate(face, axis, ng):
    """Cell values of a face field by the centred face -> cell rational
    stencil (mhd_staggering.hpp:77-112) where it fits in the padded array;
    NaN elsewhere."""
    w, den = _F2C[2 * ng]
    W = len(w)
    out = np.full_like(face, np.nan)
    n = face.shape[1 - axis]
    for c in range(W // 2 - 1, n - W // 2):
        acc = 0.0
        for k in range(W):
            q = c - (W // 2 - 1) + k
            acc = acc + w[k] * (face[:, q] if axis == 0 else face[q, :])
        if axis == 0:
            out[:, c] = acc / den
        else:
            out[c, :] = acc / den
    return out


def _assemble_faces(rho, vx, vy, vz, p, bx_face, by_face, bz, gamma, ng):
    """Conserved arrays with the face field; the magnetic energy uses the
    collocated cell field the solver itself reads back, so that the gas
    pressure is the intended p (the reference recollocates the magnetic
    energy when seeding, mhd_initial_conditions.hip:222-340)."""
    bxc = _collocate(bx_face, 0, ng)
    byc = _collocate(by_face, 1, ng)
    kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    mag = 0.5 * (bxc * bxc + byc * byc + bz * bz)
    near = 0.5 * (0.25 * (bx_face + np.roll(bx_face, -1, 1)) ** 2 +
                  0.25 * (by_face + np.roll(by_face, -1, 0)) ** 2 + bz * bz)
    energy = p / (gamma - 1.0) + kin + np.where(np.isfinite(mag), mag, near)
    return [np.ascontiguousarray(a, dtype=np.float64) for a in
            (rho, rho * vx, rho * vy, rho * vz, energy, bx_face, by_face, bz)]


OBLIQUE_H = 2.0 ** -9
_QB = 2.0 ** -35  # lattice of field values


def _lattice_faces(a, b, Ap, nx, ny, ng, h=OBLIQUE_H):
    """Faces of B = (b, -a) + curl(Ap z) with Ap periodic on the box
    (nx h) x (ny h): Ap is sampled at the wrapped corner positions."""
    ii = np.arange(-ng, nx + ng + 1)
    jj = np.arange(-ng, ny + ng + 1)
    XC, YC = np.meshgrid((ii % nx) * h, (jj % ny) * h, indexing="xy")
    A = np.rint(Ap(XC, YC) / (_QB * h))  # integer multiples of q
    bq = float(np.rint(b / _QB)) * _QB
    aq = float(np.rint(a / _QB)) * _QB
    bx = bq + (A[1:, :-1] - A[:-1, :-1]) * _QB
    by = -aq - (A[:-1, 1:] - A[:-1, :-1]) * _QB
    return np.ascontiguousarray(bx), np.ascontiguousarray(by)


def oblique_modes(angle, lx, ly, kmax=4):
    """Wave numbers (l, m) along x and y, 0..kmax, whose direction
    atan2(m/ly, l/lx) is closest to `angle`; the pattern is then periodic."""
    best = None
    for l in range(kmax + 1):
        for m in range(kmax + 1):
            if l == 0 and m == 0:
                continue
            th = math.atan2(m / ly, l / lx)
            d = abs(th - angle)
            if best is None or d < best[0] - 1e-12:
                best = (d, l, m)
    return best[1], best[2]


def _oblique_frame(n, ny, angle):
    lx, ly = n * OBLIQUE_H, ny * OBLIQUE_H
    l, m = oblique_modes(angle, lx, ly)
    kx, ky = l / lx, m / ly
    lam = 1.0 / math.hypot(kx, ky)
    c, s_ = kx * lam, ky * lam
    return lx, ly, kx, ky, lam, c, s_


def brio_wu_rotated(n, ny=None, order=5, angle=0.0, gamma=2.0, bn=0.75, bt=1.0):
    """Brio-Wu states (rho 1 | 0.125, p 1 | 0.1, B_n = 0.75, B_t = +1 | -1,
    gamma 2) as a periodic double shock tube: the left state fills the band
    1/4 <= frac(phase) < 3/4 of a plane pattern whose normal is the closest
    commensurate direction to `angle` (oblique_modes) on the exact lattice
    box (n h) x (ny h).  Outflow ghosts of an oblique tube would copy a field
    that the cell collocation no longer matches, so the tube is periodic.
    Returns (arrays, lx, ly, angle used)."""
    ny = n if ny is None else ny
    ng = nghost(order)
    lx, ly, kx, ky, lam, c, s_ = _oblique_frame(n, ny, angle)

    def G(f):  # integral of B_t over the normal coordinate, per unit phase
        return np.where(f < 0.25, -bt * f,
                        np.where(f < 0.75, -0.25 * bt + bt * (f - 0.25),
                                 0.25 * bt - bt * (f - 0.75)))

    def Ap(x, y):
        ph = kx * x + ky * y
        return -lam * G(ph - np.floor(ph))

    bx, by = _lattice_faces(-bn * s_, bn * c, Ap, n, ny, ng)
    X, Y = np.meshgrid(_centres(n, ng, lx), _centres(ny, ng, ly), indexing="xy")
    ph = kx * X + ky * Y
    f = ph - np.floor(ph)
    left = (f >= 0.25) & (f < 0.75)
    rho = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros_like(X)
    return (_assemble_faces(rho, z, z, z, p, bx, by, z, gamma, ng), lx, ly,
            math.atan2(s_, c))


def _wave_eigenvector(kind, rho, p, bn, bt1, bt2, gamma):
    """Right eigenvector of the 1-D primitive Jacobian (rho, vn, vt1, vt2, p,
    bt1, bt2) at rest for the right-going fast or Alfven wave."""
    J = np.zeros((7, 7))
    J[0, 1] = rho
    J[1, 4], J[1, 5], J[1, 6] = 1.0 / rho, bt1 / rho, bt2 / rho
    J[2, 5] = -bn / rho
    J[3, 6] = -bn / rho
    J[4, 1] = gamma * p
    J[5, 1], J[5, 2] = bt1, -bn
    J[6, 1], J[6, 3] = bt2, -bn
    w, V = np.linalg.eig(J)
    w, V = w.real, V.real
    if kind == "fast":
        k = int(np.argmax(w))
    else:
        ca = abs(bn) / math.sqrt(rho)
        k = int(np.argmin(np.abs(w - ca)))
    r = V[:, k]
    return r / np.max(np.abs(r)), float(w[k])


def linear_wave(n, ny=None, order=5, angle=math.pi / 4, kind="fast", amplitude=1e-6,
                gamma=5.0 / 3.0):
    """Linear fast or Alfven wave, one wavelength per commensurate period of
    the exact lattice box (n h) x (ny h) along the direction closest to
    `angle`; background rho=1, p=1/gamma, wave-frame B = (1, sqrt 2, 1/2).
    Returns (arrays, lx, ly, angle used)."""
    ny = n if ny is None else ny
    ng = nghost(order)
    lx, ly, kx, ky, lam, c, s_ = _oblique_frame(n, ny, angle)
    rho0, p0, bn, b1, b2 = 1.0, 1.0 / gamma, 1.0, math.sqrt(2.0), 0.5
    r, _ = _wave_eigenvector(kind, rho0, p0, bn, b1, b2, gamma)
    two_pi = 2.0 * math.pi

    def Ap(x, y):
        return -amplitude * r[5] * lam * np.sin(two_pi * (kx * x + ky * y)) / two_pi

    bx, by = _lattice_faces(-bn * s_ - b1 * c, bn * c - b1 * s_, Ap, n, ny, ng)
    X, Y = np.meshgrid(_centres(n, ng, lx), _centres(ny, ng, ly), indexing="xy")
    ph = amplitude * np.cos(two_pi * (kx * X + ky * Y))
    rho = rho0 + r[0] * ph
    vn, vt1, vt2 = r[1] * ph, r[2] * ph, r[3] * ph
    p = p0 + r[4] * ph
    bz = b2 + r[6] * ph
    vx, vy = vn * c - vt1 * s_, vn * s_ + vt1 * c
    return (_assemble_faces(rho, vx, vy, vt2, p, bx, by, bz, gamma, ng), lx, ly,
            math.atan2(s_, c))


GENERATORS = {"orszag_tang": orszag_tang, "rotor": rotor, "blast": blast}


def batch_instances(count=256, seed=0, lo=64, hi=512, order=5):
    """The seeded batch of independent instances: sides log-uniform in
    [lo, hi] per axis; family uniform over Orszag-Tang (amplitude U[0.5, 2],
    periodic, unit box), rotated Brio-Wu (angle U[0, pi/2), gamma 2, periodic
    double tube) and a linear fast or Alfven wave (amplitude 1e-6, angle
    U[0, pi/2), periodic); the oblique families live on the exact lattice box
    (nx h) x (ny h) with the commensurate direction closest to the drawn
    angle.
    Returns dicts with family, nx, ny, lx, ly, gamma, bc (0 periodic,
    1 outflow) and a zero-argument `arrays` callable."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        nx = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        ny = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        fam = int(rng.integers(0, 3))
        if fam == 0:
            amp = float(rng.uniform(0.5, 2.0))
            out.append(dict(family="orszag_tang", nx=nx, ny=ny, lx=1.0, ly=1.0,
                            gamma=5.0 / 3.0, bc=0, amplitude=amp,
                            arrays=lambda nx=nx, ny=ny, amp=amp: orszag_tang(
                                nx, order=order, amplitude=amp, ny=ny)))
        elif fam == 1:
            ang = float(rng.uniform(0.0, math.pi / 2))
            out.append(dict(family="brio_wu", nx=nx, ny=ny, lx=nx * OBLIQUE_H,
                            ly=ny * OBLIQUE_H, gamma=2.0, bc=0, angle=ang,
                            arrays=lambda nx=nx, ny=ny, ang=ang: brio_wu_rotated(
                                nx, ny, order=order, angle=ang)[0]))
        else:
            ang = float(rng.uniform(0.0, math.pi / 2))
            kind = "fast" if rng.integers(0, 2) == 0 else "alfven"
            out.append(dict(family=f"{kind}_wave", nx=nx, ny=ny, lx=nx * OBLIQUE_H,
                            ly=ny * OBLIQUE_H, gamma=5.0 / 3.0, bc=0, angle=ang,
                            arrays=lambda nx=nx, ny=ny, ang=ang, kind=kind: linear_wave(
                                nx, ny, order=order, angle=ang, kind=kind)[0]))
    return out


def training_runs(count=12, seed=1, n=512, order=5):
    """Seeded plain-method runs for the indicator's training labels: rotor
    (radius log-uniform in [0.05, 0.2], field log-uniform in [0.1, 10]),
    blast (radius in [0.05, 0.2], pressure ratio in [10, 1000], field in
    [0.1, 10]) and Orszag-Tang (field scale in [0.1, 10] as amplitude of B^2
    relative to the gas), cycled in that order.  Returns dicts with family,
    parameters, bc, a step budget that reaches the developed flow, and a
    zero-argument `arrays` callable."""
    rng = np.random.default_rng(seed)
    lu = lambda a, b: float(math.exp(rng.uniform(math.log(a), math.log(b))))  # noqa: E731
    out = []
    for k in range(count):
        fam = ("rotor", "blast", "orszag_tang")[k % 3]
        scale = n / 512.0  # steps to a comparable time at this resolution
        if fam == "rotor":
            r0, bf = lu(0.05, 0.2), lu(0.1, 10.0)
            out.append(dict(family=fam, radius=r0, field=bf, bc=1, steps=int(1200 * scale),
                            arrays=lambda r0=r0, bf=bf: rotor(n, order=order, r0=r0, bx=bf)))
        elif fam == "blast":
            r0, ratio, bf = lu(0.05, 0.2), lu(10.0, 1000.0), lu(0.1, 10.0)
            out.append(dict(family=fam, radius=r0, ratio=ratio, field=bf, bc=1,
                            steps=int(1200 * scale),
                            arrays=lambda r0=r0, ratio=ratio, bf=bf: blast(
                                n, order=order, radius=r0, p_in=0.1 * ratio, p_out=0.1,
                                b=bf / math.sqrt(2.0))))
        else:
            amp = lu(0.1, 10.0)
            out.append(dict(family=fam, field=amp, bc=0, steps=int(4000 * scale),
                            arrays=lambda amp=amp: _ot_field_scaled(n, order, amp)))
    return out


def _ot_field_scaled(n, order, scale):
    """Orszag-Tang with the magnetic field scaled by sqrt(scale) at fixed gas
    state (plasma beta divided by `scale`)."""
    arr = orszag_tang(n, order=order)
    ng = nghost(order)
    out = list(arr)
    f = math.sqrt(scale)
    bx, by = arr[5] * f, arr[6] * f
    # energy: gas + kinetic unchanged, magnetic energy of the scaled field
    old_mag = 0.5 * (arr[5] ** 2 + arr[6] ** 2)
    out[4] = np.ascontiguousarray(arr[4] - old_mag + 0.5 * (bx ** 2 + by ** 2))
    out[5], out[6] = np.ascontiguousarray(bx), np.ascontiguousarray(by)
    return out


def combined_instances(seed=2, count=64, lo=256, hi=1024, order=7, ot_n=8192):
    """The large combined batch: one Orszag-Tang instance at ot_n^2 and
    `count` rotor / blast instances (alternating) with square sides
    log-uniform in [lo, hi] and radii log-uniform in [0.05, 0.2], outflow.
    Returns dicts like batch_instances."""
    rng = np.random.default_rng(seed)
    out = [dict(family="orszag_tang", nx=ot_n, ny=ot_n, lx=1.0, ly=1.0, gamma=5.0 / 3.0, bc=0,
                arrays=lambda: orszag_tang(ot_n, order=order))]
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        r0 = float(math.exp(rng.uniform(math.log(0.05), math.log(0.2))))
        if k % 2 == 0:
            out.append(dict(family="rotor", nx=n, ny=n, lx=1.0, ly=1.0, gamma=5.0 / 3.0, bc=1,
                            radius=r0, arrays=lambda n=n, r0=r0: rotor(n, order=order, r0=r0)))
        else:
            out.append(dict(family="blast", nx=n, ny=n, lx=1.0, ly=1.0, gamma=5.0 / 3.0, bc=1,
                            radius=r0, arrays=lambda n=n, r0=r0: blast(n, order=order, radius=r0)))
    return out
