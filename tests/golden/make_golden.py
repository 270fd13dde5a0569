"""Generate the golden fixtures of tests/golden/ by running the reference's OWN
MHD solver built for the CPU (oracle/build_ref.sh -> oracle/_ref).

    python tests/golden/make_golden.py short     # few-step fixtures (seconds)
    python tests/golden/make_golden.py ot_t05    # OT 128^2 MP5 to t=0.5 (long)
    python tests/golden/make_golden.py large     # rotor / blast 512^2 MP7 (minutes)

Fixtures hold the seeded initial state's generator parameters, the dt of
every step and the reference state after the last step, so GPU tests can pin
the CUDA product against the reference where the reference itself cannot run.
The 512^2 fixtures (the benchmark's rotor and blast workloads at MP7) keep
the state in summary form to stay small: per component, over its evolved
region, the signed and absolute sums of every row and column, and every 8th
value of every 8th row.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import mhd_cases as M  # noqa: E402

SHORT = [
    # name, case, n, order, bc, steps
    ("ot32_mp5", "ot", 32, 5, M.PERIODIC, 6),
    ("ot32_mp7", "ot", 32, 7, M.PERIODIC, 4),
    ("rotor32_mp7", "rotor", 32, 7, M.OUTFLOW, 6),
    ("blast32_mp7", "blast", 32, 7, M.OUTFLOW, 6),
    ("rotor48_mp5", "rotor", 48, 5, M.OUTFLOW, 4),
    ("ot24_muscl", "ot", 24, 2, M.PERIODIC, 5),
]
CASES = {"ot": M.orszag_tang, "rotor": M.rotor, "blast": M.blast}


LARGE = [
    ("rotor512_mp7", "rotor", 512, 7, M.OUTFLOW, 2),
    ("blast512_mp7", "blast", 512, 7, M.OUTFLOW, 2),
]
SUB = 8  # subsample stride of the summary fixtures


def summarize(st, ng, n):
    """Per component, over its evolved region (interior cells, plus the owned
    high faces of the face fields): signed and absolute sums of every row and
    column, and every SUB-th value of every SUB-th row."""
    out = {}
    for c, name in enumerate(M.COMPONENTS):
        a = M._evolved(st[c], c, ng, n, n)
        out[name + "_row_sum"] = a.sum(axis=1)
        out[name + "_row_abs"] = np.abs(a).sum(axis=1)
        out[name + "_col_sum"] = a.sum(axis=0)
        out[name + "_col_abs"] = np.abs(a).sum(axis=0)
        out[name + "_sub"] = a[::SUB, ::SUB].copy()
    return out


def run(name, case, n, order, bc, steps=None, t_end=None, keep="all"):
    R = M.RefLib()
    s = R.solver(n, n, order, bc=bc)
    s.seed(CASES[case](n, order=order))
    dts, t, t0 = [], 0.0, time.time()
    k = 0
    while True:
        if steps is not None and k >= steps:
            break
        if t_end is not None and not t < t_end:
            break
        dt = s.cfl()
        if t_end is not None:
            rem = t_end - t
            dt = min(dt, rem)
        s.step(dt)
        t = t_end if (t_end is not None and dt == t_end - t) else t + dt
        dts.append(dt)
        k += 1
        if k % 100 == 0:
            print(f"{name}: step {k} t={t:.6f} ({time.time() - t0:.0f}s)", flush=True)
    st = s.read()
    d = ctypes_divb(R, s)
    payload = dict(case=case, n=n, order=order, bc=np.array(bc), dts=np.array(dts), t=t, divb=d)
    if keep == "summary":
        payload.update(summarize(st, M.nghost(order), n), sub_stride=SUB)
    else:
        comps = range(8) if keep == "all" else [0]
        for c in comps:
            payload[M.COMPONENTS[c]] = st[c]
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **payload)
    print(f"{name}: {k} steps t={t:.6g} divb={d:.3e} ({time.time() - t0:.1f}s)")


def ctypes_divb(R, s):
    import ctypes
    d = ctypes.c_double()
    R.lib.qref_divb(s.h, ctypes.byref(d))
    return d.value


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "short"
    if what == "short":
        for row in SHORT:
            run(*row)
    elif what == "ot_t05":
        run("ot128_mp5_t05", "ot", 128, 5, M.PERIODIC, t_end=0.5, keep="rho")
    elif what == "large":
        for row in LARGE:
            run(*row, keep="summary")
