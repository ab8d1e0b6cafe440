"""wake_b200 - B200-native lattice-Boltzmann time step for wake.

The compute lives in libwake_b200.so (hand-written sm_100a CUDA behind the C
ABI of include/wake_gpu.h). This package is a thin Python mirror of the
reference's host classes over that ABI; it never computes on the CPU.
"""
from ._lib import EXPORTED, LIB_PATH, WakeError, addr, check, lib
from .analytics import FieldAnalytics, VtkExporter
from .grid import (BGK, FLUID, INFLOW, MOVING_WALL, MRT, OUTFLOW, SOLID, TRT, LatticeGrid2D, LatticeGrid3D,
                   LatticeGrid3DQ27)

__all__ = [
    "lib", "check", "addr", "WakeError", "EXPORTED", "LIB_PATH",
    "LatticeGrid2D", "LatticeGrid3D", "LatticeGrid3DQ27", "FieldAnalytics", "VtkExporter",
    "BGK", "TRT", "MRT", "FLUID", "SOLID", "INFLOW", "OUTFLOW", "MOVING_WALL",
]


def strouhal_frequency(signal, dt: float = 1.0) -> float:
    """FP64 Strouhal peak frequency of a lift history (see wake_strouhal_frequency)."""
    import numpy as np

    s = np.ascontiguousarray(signal, dtype=np.float64)
    return float(lib.wake_strouhal_frequency(addr(s), len(s), dt))
