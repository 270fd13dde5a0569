"""quasar_b200: B200-native (sm_100a) 2-D ideal-MHD finite-volume step.

The hot path (MP5/MP7 characteristic reconstruction, Gauss-point HLLD, upwind
constrained transport, SSP-RK3, CFL reduction) runs as hand-written FP64 CUDA
kernels behind the C ABI in include/quasar_mhd.h; `quasar_b200.mhd` mirrors
the reference's `_core.mhd` Python module on top of it.
"""
from . import mhd  # noqa: F401
from .mhd import Grid2D, MhdBoundarySpec, MhdConfig, MhdSolver2D  # noqa: F401

__all__ = ["mhd", "Grid2D", "MhdBoundarySpec", "MhdConfig", "MhdSolver2D"]
