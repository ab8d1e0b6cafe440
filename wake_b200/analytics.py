"""Field analytics and VTK export of a lattice's state.

``FieldAnalytics`` keeps the static methods of wake::FieldAnalytics
(include/wake/analytics/field_analytics.hpp:10-26) and ``VtkExporter`` those of
wake::VtkExporter (include/wake/export/vtk_exporter.hpp:9-36). The vorticity and
Q-criterion are computed on the GPU from the grid's resident moments; the VTK
files are written by the library's host writer in the reference's bytes.
"""
from __future__ import annotations

import os

import numpy as np

from ._lib import addr, check, lib


def _out(n: int, out, device: bool):
    if out is not None:
        return out
    if device:
        import torch

        return torch.empty(n, dtype=torch.float32, device="cuda")
    return np.empty(n, dtype=np.float32)


class FieldAnalytics:
    """GPU counterpart of wake::FieldAnalytics (src/analytics/field_analytics.cpp:18-63)."""

    @staticmethod
    def compute_vorticity(grid, vorticity_out=None, device: bool = False):
        """omega_z = d(uy)/dx - d(ux)/dy of a D2Q9 grid's current state (numpy, or a CUDA tensor with device=True)."""
        out = _out(grid.total_nodes(), vorticity_out, device)
        check(lib.wake_grid_compute_vorticity(grid.handle, addr(out)))
        return out

    @staticmethod
    def compute_3d_features(grid, omega_x_out=None, omega_y_out=None, omega_z_out=None, q_criterion_out=None,
                            device: bool = False):
        """(omega_x, omega_y, omega_z, Q) of a 3D grid's current state."""
        n = grid.total_nodes()
        outs = [_out(n, o, device) for o in (omega_x_out, omega_y_out, omega_z_out, q_criterion_out)]
        check(lib.wake_grid_compute_3d_features(grid.handle, *[addr(o) for o in outs]))
        return tuple(outs)

    @staticmethod
    def compute_max_vorticity_2d(vorticity) -> float:
        """Largest |value| of a vorticity array (host array or CUDA tensor); NaN values are skipped."""
        import ctypes as C

        v = vorticity
        if not hasattr(v, "data_ptr"):
            v = np.ascontiguousarray(v, dtype=np.float32).ravel()
            n = v.size
        else:
            if v.dtype.itemsize != 4 or not v.is_contiguous():
                raise ValueError("vorticity must be a contiguous float32 tensor")
            n = v.numel()
        m = C.c_float()
        check(lib.wake_field_abs_max(addr(v), n, C.addressof(m)))
        return m.value

    @staticmethod
    def max_vorticity(grid) -> float:
        """compute_vorticity + compute_max_vorticity_2d of a D2Q9 grid, on the device."""
        import ctypes as C

        m = C.c_float()
        check(lib.wake_grid_max_vorticity(grid.handle, C.addressof(m)))
        return m.value


def _host(a, n, dtype=np.float32):
    if a is None:
        return None
    if hasattr(a, "detach"):
        a = a.detach().cpu().numpy()
    a = np.ascontiguousarray(a, dtype=dtype).ravel()
    if a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class VtkExporter:
    """wake::VtkExporter (src/export/vtk_exporter.cpp:8-223): same files, same bytes."""

    @staticmethod
    def export_vti_2d(filepath, grid, vorticity=None, threads: int = 0) -> bool:
        """Velocity, Speed, Density, optional Vorticity and CellType of a D2Q9 grid's current state."""
        m = grid.macroscopic()
        n = grid.total_nodes()
        t = grid.cell_type_data()
        v = _host(vorticity, n)
        rc = lib.wake_vtk_write_vti_2d(os.fsencode(filepath), grid.nx, grid.ny, addr(m["ux"]), addr(m["uy"]),
                                       addr(m["speed"]), addr(m["rho"]), addr(v), addr(t), threads)
        return rc == 0

    @staticmethod
    def export_vti_3d(filepath, grid, q_criterion=None, vorticity=None, threads: int = 0) -> bool:
        """Velocity, Speed, Density, optional Q_Criterion and Vorticity (a (3, n) array, an (n, 3) array or
        three arrays) and CellType of a 3D grid's current state."""
        m = grid.macroscopic()
        n = grid.total_nodes()
        t = grid.cell_type_data()
        qc = _host(q_criterion, n)
        comps = [None, None, None]
        if vorticity is not None:
            if isinstance(vorticity, (tuple, list)):
                comps = [_host(c, n) for c in vorticity]
            else:
                a = vorticity.detach().cpu().numpy() if hasattr(vorticity, "detach") else np.asarray(vorticity)
                a = a.reshape(3, n) if a.shape[0] == 3 and a.size == 3 * n else a.reshape(n, 3).T
                comps = [_host(a[i], n) for i in range(3)]
        rc = lib.wake_vtk_write_vti_3d(os.fsencode(filepath), grid.nx, grid.ny, grid.nz, addr(m["ux"]),
                                       addr(m["uy"]), addr(m["uz"]), addr(m["speed"]), addr(m["rho"]), addr(qc),
                                       *[addr(c) for c in comps], addr(t), threads)
        return rc == 0

    @staticmethod
    def export_grid(filepath, grid, analytics: bool = True, threads: int = 0) -> None:
        """The grid's state in one call: moments, cell types and the device-computed vorticity (2D) or
        vorticity + Q-criterion (3D)."""
        check(lib.wake_grid_export_vti(grid.handle, os.fsencode(filepath), int(analytics), threads))

    @staticmethod
    def write_pvd_manifest(manifest_path, file_prefix, start_step, end_step, step_interval, dt=1.0) -> bool:
        rc = lib.wake_vtk_write_pvd(os.fsencode(manifest_path), os.fsencode(file_prefix), start_step, end_step,
                                    step_interval, dt)
        return rc == 0
