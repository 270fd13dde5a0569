"""Learned troubled-cell indicator (include/quasar_mhd_indicator.h)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native

FEATURES = 200
HIDDEN = 64
PARAMS = HIDDEN * FEATURES + HIDDEN + HIDDEN * HIDDEN + HIDDEN + HIDDEN + 1


class TroubledCellIndicator:
    """200 -> 64 -> 64 -> 1 GELU network on the tensor cores (no reference
    counterpart; trained on the reference limiter's own firing decisions)."""

    def __init__(self, seed: int = 0):
        h = ctypes.c_void_p()
        _native.check(_native.lib().qmhd_indicator_create(ctypes.c_ulonglong(seed), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _native.lib().qmhd_indicator_destroy(h)
            self._h = None

    def params(self) -> np.ndarray:
        out = np.empty(PARAMS, dtype=np.float32)
        _native.check(_native.lib().qmhd_indicator_get_params(self._h, out.ctypes.data, PARAMS))
        return out

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(np.asarray(p, dtype=np.float32).reshape(-1))
        _native.check(_native.lib().qmhd_indicator_set_params(self._h, a.ctypes.data, a.size))

    def forward(self, features) -> np.ndarray:
        x = np.ascontiguousarray(np.asarray(features, dtype=np.float32).reshape(-1, FEATURES))
        out = np.empty(len(x), dtype=np.float32)
        _native.check(_native.lib().qmhd_indicator_forward(self._h, x.ctypes.data, len(x),
                                                           out.ctypes.data))
        return out

    def gradient(self, features, labels, pos_weight: float = 1.0):
        """(mean weighted BCE, gradient) of host rows from the tensor-core
        backward pass; no update."""
        x = np.ascontiguousarray(np.asarray(features, dtype=np.float32).reshape(-1, FEATURES))
        y = np.ascontiguousarray(np.asarray(labels, dtype=np.uint8).reshape(-1))
        g = np.empty(PARAMS, dtype=np.float32)
        loss = ctypes.c_double()
        _native.check(_native.lib().qmhd_indicator_gradient(
            self._h, x.ctypes.data, y.ctypes.data, len(x), ctypes.c_float(pos_weight),
            g.ctypes.data, PARAMS, ctypes.byref(loss)))
        return loss.value, g

    def collect(self, solver, tol: float = 1e-6) -> None:
        """Append the solver's live state: features, and labels 1 where a
        limited face state departs from the unlimited component-wise one by
        more than `tol` of the state's scale (a negative tol: where the MP
        limiter fired on any characteristic field, the literal label)."""
        _native.check(_native.lib().qmhd_indicator_collect(self._h, solver._h, ctypes.c_float(tol)))

    def rows(self) -> int:
        return int(_native.lib().qmhd_indicator_rows(self._h))

    def labels(self) -> np.ndarray:
        """The collected labels, one per row in collection order (per state
        its interior cells row by row)."""
        out = np.empty(self.rows(), dtype=np.uint8)
        _native.check(_native.lib().qmhd_indicator_labels(self._h, out.ctypes.data, out.size))
        return out

    def clear(self) -> None:
        _native.check(_native.lib().qmhd_indicator_clear(self._h))

    def train(self, epochs=2, tiles_per_step=256, lr=1e-3, pos_weight=4.0, holdout=20, seed=0):
        loss = ctypes.c_double()
        _native.check(_native.lib().qmhd_indicator_train(
            self._h, int(epochs), int(tiles_per_step), ctypes.c_float(lr),
            ctypes.c_float(pos_weight), int(holdout), ctypes.c_ulonglong(seed), ctypes.byref(loss)))
        return loss.value

    def evaluate(self, threshold: float, holdout: int = 20):
        r, f = ctypes.c_double(), ctypes.c_double()
        p, t = ctypes.c_longlong(), ctypes.c_longlong()
        _native.check(_native.lib().qmhd_indicator_evaluate(
            self._h, ctypes.c_float(threshold), int(holdout), ctypes.byref(r), ctypes.byref(f),
            ctypes.byref(p), ctypes.byref(t)))
        return dict(recall=r.value, flagged=f.value, positives=p.value, total=t.value)

    def threshold_for_recall(self, recall: float, holdout: int = 20) -> float:
        t = ctypes.c_float()
        _native.check(_native.lib().qmhd_indicator_threshold_for_recall(
            self._h, ctypes.c_double(recall), int(holdout), ctypes.byref(t)))
        return t.value

    def attach(self, solver, threshold: float) -> None:
        """Run `solver` in learned mode with this indicator (kept alive by
        the solver object)."""
        _native.check(_native.lib().qmhd_solver_set_indicator(solver._h, self._h,
                                                              ctypes.c_float(threshold)))
        solver._indicator = self


def attach_batch(ind, batch, threshold: float) -> None:
    """Learned mode for every instance of an MhdBatch2D (kept alive by it)."""
    _native.check(_native.lib().qmhd_batch_set_indicator(batch._h, ind._h,
                                                         ctypes.c_float(threshold)))
    batch._indicator = ind


def detach(solver) -> None:
    """Back to the plain step."""
    _native.check(_native.lib().qmhd_solver_set_indicator(solver._h, None, ctypes.c_float(0.0)))
    solver._indicator = None


def learned_face_counts(solver):
    a, b = ctypes.c_longlong(), ctypes.c_longlong()
    _native.check(_native.lib().qmhd_solver_learned_face_counts(solver._h, ctypes.byref(a),
                                                                ctypes.byref(b)))
    return a.value, b.value
