"""Telemetry files in the reference's formats (C ABI ``wake_telemetry_*``).

``TelemetryExporter`` mirrors wake::TelemetryExporter
(include/wake/export/csv_telemetry.hpp, src/export/csv_telemetry.cpp:21-125):
the aerodynamic CSV, the performance CSV and the summary JSON come out byte for
byte as the reference writes them, so its scripts read them unchanged.
``record_history`` converts a grid's per-step FP64 force history
(``LatticeGrid2D.force_history()``) into the records a scenario would have made.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._lib import addr, check, lib


class TelemetryExporter:
    def __init__(self):
        self._h = lib.wake_telemetry_create()

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.wake_telemetry_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def record_aero(self, step: int, time: float, fx: float, fy: float, fz: float = 0.0, torque_z: float = 0.0,
                    rho_inf: float = 1.0, u_inf: float = 0.05, area: float = 1.0, chord: float = 1.0) -> None:
        """One sample; coefficients as compute_aerodynamic_coefficients (float arithmetic)."""
        check(lib.wake_telemetry_record_aero(self._h, step, time, fx, fy, fz, torque_z, rho_inf, u_inf, area, chord))

    def record_history(self, history, first_step: int = 1, every: int = 10, is3d: bool = False,
                       rho_inf: float = 1.0, u_inf: float = 0.05, area: float = 1.0, chord: float = 1.0) -> None:
        """Rows of a force history [n, 3] for steps first_step, first_step + 1, ...; the steps
        divisible by `every` become records (the scenarios record every 10th step)."""
        h = np.ascontiguousarray(history, np.float64).reshape(-1, 3)
        check(lib.wake_telemetry_record_history(self._h, addr(h), h.shape[0], first_step, every, int(is3d), rho_inf,
                                                u_inf, area, chord))

    def record_performance(self, step: int, step_time_ms: float, mlups: float, max_speed: float = 0.0,
                           total_mass: float = 0.0, kinetic_energy: float = 0.0) -> None:
        check(lib.wake_telemetry_record_performance(self._h, step, step_time_ms, mlups, max_speed, total_mass,
                                                    kinetic_energy))

    def clear(self) -> None:
        lib.wake_telemetry_clear(self._h)

    def aero_count(self) -> int:
        return check(lib.wake_telemetry_count(self._h, 0))

    def coefficients(self) -> np.ndarray:
        """[n, 3] float32 (cd, cl, cm) of the aerodynamic records."""
        n = self.aero_count()
        out = np.zeros((n, 3), np.float32)
        buf = (ctypes.c_float * 3)()
        for i in range(n):
            check(lib.wake_telemetry_get_coefficients(self._h, i, ctypes.addressof(buf)))
            out[i] = buf[:]
        return out

    def write_aero_csv(self, path) -> None:
        check(lib.wake_telemetry_write_aero_csv(self._h, str(path).encode()))

    def write_performance_csv(self, path) -> None:
        check(lib.wake_telemetry_write_performance_csv(self._h, str(path).encode()))

    def write_summary_json(self, path, simulation_name: str, strouhal_number: float = 0.0,
                           shedding_frequency: float = 0.0) -> None:
        check(lib.wake_telemetry_write_summary_json(self._h, str(path).encode(), simulation_name.encode(),
                                                    strouhal_number, shedding_frequency))
