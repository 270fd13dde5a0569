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
