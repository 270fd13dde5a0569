"""Train the troubled-cell indicator on the GPU and write its parameters.

    python -m quasar_b200.train_indicator --out quasar_b200/data/indicator_mp5.npz

Labels come from plain-method runs of the seeded rotor / blast / Orszag-Tang
families of `quasar_b200.ics.training_runs`: evenly spaced live states of
each run are collected (features of every interior cell and whether
its limited characteristic face states depart from the component-wise
unlimited ones), then Adam trains the network with the tensor-core
forward/backward kernels.  The threshold is the smallest logit that keeps
`recall` of the held-out limiter activations.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import ics, mhd
from .indicator import TroubledCellIndicator


def _solver(n, order, bc):
    cfg = mhd.MhdConfig()
    cfg.grid = mhd.Grid2D(n, n, 1.0, 1.0)
    cfg.reconstruction = "mp5" if order == 5 else "mp7"
    side = "periodic" if bc == 0 else "outflow"
    cfg.boundary = mhd.MhdBoundarySpec([side] * 4, [side] * 4)
    return mhd.MhdSolver2D(cfg)


def collect(ind, n=512, runs=12, snapshots=20, order=5, seed=1, tol=1e-6, log=print):
    """Step each seeded run through its step budget, collecting `snapshots`
    evenly spaced live states."""
    t0 = time.time()
    for k, run in enumerate(ics.training_runs(count=runs, seed=seed, n=n, order=order)):
        s = _solver(n, order, run["bc"])
        for name, a in zip(ics.COMPONENTS, run["arrays"]()):
            s.seed_state(name, a)
        t, done = 0.0, 0
        steps, every = run["steps"], max(1, run["steps"] // snapshots)
        while done < steps:
            try:
                t, taken = s.advance_auto(t, 1e30, every)
            except RuntimeError as e:  # a run the plain method cannot continue ends here
                log(f"run {k} ({run['family']}) stops after {done} steps: {e}")
                break
            done += taken
            ind.collect(s, tol)
        log(f"run {k} {run['family']}: {done} steps, rows {ind.rows()} ({time.time() - t0:.0f}s)")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--runs", type=int, default=12)
    ap.add_argument("--snapshots", type=int, default=20)
    ap.add_argument("--order", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--tiles", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--pos-weight", type=float, default=30.0)
    ap.add_argument("--recall", type=float, default=0.95)
    ap.add_argument("--holdout", type=int, default=20)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--tol", type=float, default=1e-4)
    a = ap.parse_args(argv)
    a.out = a.out or default_path(a.order)
    ind = TroubledCellIndicator(seed=a.seed)
    collect(ind, a.n, a.runs, a.snapshots, a.order, a.seed, a.tol)
    t0 = time.time()
    losses = []
    for ep in range(a.epochs):
        lr = a.lr * (0.5 ** (ep // max(1, a.epochs // 3)))
        losses.append(ind.train(epochs=1, tiles_per_step=a.tiles, lr=lr, pos_weight=a.pos_weight,
                                holdout=a.holdout, seed=a.seed + ep))
        print(f"epoch {ep + 1}: loss {losses[-1]:.5f} lr {lr:.2e} ({time.time() - t0:.1f}s)")
    thr = ind.threshold_for_recall(a.recall, a.holdout)
    ev = ind.evaluate(thr, a.holdout)
    print(f"threshold {thr:.4f}: held-out recall {ev['recall']:.4f}, flagged {ev['flagged']:.4f}, "
          f"positives {ev['positives']} of {ev['total']}")
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    meta = dict(vars(a), rows=ind.rows(), losses=losses, threshold=thr, **ev)
    np.savez(a.out, params=ind.params(), threshold=np.float32(thr), meta=json.dumps(meta))
    return ind, thr, ev


def inference_report(n=2048, order=5, t_develop=0.3, steps=100, snapshots=2, path=None):
    """The indicator at inference on Orszag-Tang n^2 (periodic, FP64 state).
    Two solvers advance the plain step bit for bit to t_develop (the shocks
    have formed); then one runs in learned mode and both take `steps` more
    steps with the plain run's dt.  Returns the density L1 gap (relative,
    interior), the recall of the plain run's own limiter activations by the
    flags (labels at the tolerance the weights were trained with, on
    `snapshots` evenly spaced plain states of that window) with the fraction
    of cells flagged, and the mean fraction of faces that took the
    characteristic path."""
    from .indicator import learned_face_counts
    ind, thr = load(path, order)
    z = np.load(path or default_path(order))
    tol = float(json.loads(str(z["meta"])).get("tol", 1e-4))
    solvers = []
    for _ in range(2):
        s = _solver(n, order, 0)
        for name, arr in zip(ics.COMPONENTS, ics.orszag_tang(n, order=order)):
            s.seed_state(name, arr)
        t, taken = s.advance_auto(0.0, t_develop, 10 ** 7)
        solvers.append(s)
    plain, learned = solvers
    ind.attach(learned, thr)
    probe = TroubledCellIndicator(seed=0)
    probe.set_params(ind.params())
    ng = ics.nghost(order)
    universe = 2.0 * (n + 1) * (n + 2 * ng)
    face_frac = []
    per = max(1, steps // snapshots)
    for k in range(steps):
        if k % per == 0 and k // per < snapshots:
            probe.collect(plain, tol)
        dt = plain.cfl_limit()
        plain.step_unchecked(dt)
        learned.step_unchecked(dt)
        fx, fy = learned_face_counts(learned)
        face_frac.append((fx + fy) / universe)
    ev = probe.evaluate(thr, holdout=0)
    sl = (slice(ng, ng + n), slice(ng, ng + n))
    shape = (n + 2 * ng, n + 2 * ng)
    rp = plain.state_component_to_host("rho").reshape(shape)[sl]
    rl = learned.state_component_to_host("rho").reshape(shape)[sl]
    return {"workload": f"Orszag-Tang {n}^2 MP{order}, periodic: plain to t={t:.4f} "
                        f"({taken} steps), then {steps} steps plain and learned with the "
                        "plain run's dt",
            "rho_l1_vs_plain": float(np.sum(np.abs(rl - rp)) / np.sum(np.abs(rp))),
            "limiter_recall": ev["recall"], "cells_flagged": ev["flagged"],
            "label_tol": tol, "labelled_cells": ev["total"], "limiter_positive": ev["positives"],
            "full_path_face_fraction": float(np.mean(face_frac)),
            "div_b_max": learned.divergence_b_max(), "div_b_max_plain": plain.divergence_b_max(),
            "div_b_rel": learned.divergence_b_relative(),
            "div_b_rel_plain": plain.divergence_b_relative()}


def _heuristic_scores(solver, n, order, gamma):
    """Per interior cell (row by row): the largest relative density or
    pressure jump over its 5 x 5 stencil, max |q / q_centre - 1| for
    q = rho, p -- the cheap shock detector a troubled-cell indicator must beat."""
    from numpy.lib.stride_tricks import sliding_window_view
    ng = ics.nghost(order)
    shape = (n + 2 * ng, n + 2 * ng)
    st = {c: solver.state_component_to_host(c).reshape(shape) for c in ics.COMPONENTS}
    rho = st["rho"]
    bx = 0.5 * (st["bx_face"] + np.roll(st["bx_face"], -1, axis=1))
    by = 0.5 * (st["by_face"] + np.roll(st["by_face"], -1, axis=0))
    kin = 0.5 * (st["mx"] ** 2 + st["my"] ** 2 + st["mz"] ** 2) / rho
    p = (gamma - 1.0) * (st["energy"] - kin - 0.5 * (bx * bx + by * by + st["bz_cell"] ** 2))
    sl = slice(ng - 2, ng + n + 2)
    score = np.zeros((n, n))
    for q in (rho[sl, sl], p[sl, sl]):
        win = sliding_window_view(q, (5, 5))          # (n, n, 5, 5)
        c = q[2:-2, 2:-2][:, :, None, None]
        score = np.maximum(score, np.abs(win / c - 1.0).max(axis=(2, 3)))
    return score.reshape(-1)


def _flagged_at_recall(scores, labels, recall):
    """Fraction of cells flagged by the lowest threshold on `scores` (higher
    = more troubled) that still flags `recall` of the positive labels."""
    pos = np.sort(scores[labels == 1])
    if pos.size == 0:
        return 0.0, np.inf
    thr = pos[int(np.floor((1.0 - recall) * pos.size))]
    return float(np.mean(scores >= thr)), float(thr)


def gain_report(n=512, order=5, t_develop=0.3, steps=60, recall=0.95, path=None):
    """What the trained indicator gains on a developed flow (Orszag-Tang n^2,
    plain step to t_develop): the fraction of cells each scorer must flag to
    catch `recall` of the plain limiter's activations on that state -- the
    shipped network, the same network untrained (its initial weights), and
    the density/pressure jump heuristic -- with the density L1 gap of the
    learned step at the shipped network's threshold after `steps` steps, and
    the recall of the shipped flags against the literal label (the limiter
    fired on any characteristic field) beside the training label."""
    ind, thr_shipped = load(path, order)
    z = np.load(path or default_path(order))
    tol = float(json.loads(str(z["meta"])).get("tol", 1e-4))
    gamma = 5.0 / 3.0
    solvers = []
    for _ in range(2):
        s = _solver(n, order, 0)
        for name, arr in zip(ics.COMPONENTS, ics.orszag_tang(n, order=order)):
            s.seed_state(name, arr)
        t, taken = s.advance_auto(0.0, t_develop, 10 ** 7)
        solvers.append(s)
    plain, learned = solvers
    out = {"workload": f"Orszag-Tang {n}^2 MP{order}, periodic, developed to t={t:.4f} "
                       f"({taken} plain steps)", "recall": recall, "label_tol": tol}
    trained = TroubledCellIndicator(seed=0)
    trained.set_params(ind.params())
    untrained = TroubledCellIndicator(seed=0)
    for name, net in (("trained", trained), ("untrained", untrained)):
        net.collect(plain, tol)
        thr = net.threshold_for_recall(recall, holdout=0)
        ev = net.evaluate(thr, holdout=0)
        out[name] = {"flagged": ev["flagged"], "recall": ev["recall"], "threshold": thr}
    labels = trained.labels()
    out["positives"] = int(labels.sum())
    out["cells"] = int(labels.size)
    flagged, thr = _flagged_at_recall(_heuristic_scores(plain, n, order, gamma), labels, recall)
    out["heuristic"] = {"flagged": flagged, "threshold": thr,
                        "score": "max over the 5x5 stencil of |rho/rho_c - 1| and |p/p_c - 1|"}
    # the shipped threshold on this state, against both labels
    out["shipped_threshold"] = thr_shipped
    out["shipped_recall_training_label"] = trained.evaluate(thr_shipped, holdout=0)["recall"]
    literal = TroubledCellIndicator(seed=0)
    literal.set_params(ind.params())
    literal.collect(plain, -1.0)
    lev = literal.evaluate(thr_shipped, holdout=0)
    out["literal_label"] = {"positive_fraction": lev["positives"] / max(lev["total"], 1),
                            "shipped_recall": lev["recall"], "flagged": lev["flagged"]}
    # the learned step at the shipped threshold against the plain step
    ind.attach(learned, thr_shipped)
    for _ in range(steps):
        dt = plain.cfl_limit()
        plain.step_unchecked(dt)
        learned.step_unchecked(dt)
    ng = ics.nghost(order)
    sl = (slice(ng, ng + n), slice(ng, ng + n))
    shape = (n + 2 * ng, n + 2 * ng)
    rp = plain.state_component_to_host("rho").reshape(shape)[sl]
    rl = learned.state_component_to_host("rho").reshape(shape)[sl]
    out["rho_l1_vs_plain"] = float(np.sum(np.abs(rl - rp)) / np.sum(np.abs(rp)))
    out["steps"] = steps
    return out


def default_path(order):
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", f"indicator_mp{order}.npz")


def load(path=None, order=5):
    """(indicator, threshold) from a file written by main()."""
    path = path or default_path(order)
    z = np.load(path)
    ind = TroubledCellIndicator(seed=0)
    ind.set_params(z["params"])
    return ind, float(z["threshold"])


if __name__ == "__main__":
    main()
