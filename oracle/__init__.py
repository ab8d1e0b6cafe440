"""Oracle loaders — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs use this package, and only as the checker. The product (wake_b200) never
imports it.

* ``liboracle.so`` (oracle/wake_oracle.cpp): this project's CPU restatement
  of the reference algorithm, float or double, with the extensions the
  reference lacks (applied LES, 3D Zou-He, periodic y/z, D3Q27 MRT).
* ``_ref/libwake_ref.so`` (oracle/build_ref.py): the reference's own host
  classes and mechanically translated ISPC kernels. Built only where the
  reference sources exist; travels with the tree as a prebuilt file.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libwake_ref.so"


def build_oracle() -> Path:
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)
    return ORACLE_SO


def build_reference() -> Path | None:
    from . import build_ref

    if not (build_ref.reference_dir() / "src" / "ispc").is_dir():
        return REF_SO if REF_SO.exists() else None
    return build_ref.build()


def _addr(a):
    if a is None:
        return None
    return a.ctypes.data


class Params(C.Structure):
    _fields_ = [
        ("collision", C.c_int), ("les", C.c_int), ("mrt_exact", C.c_int), ("periodic_y", C.c_int),
        ("periodic_z", C.c_int), ("inflow", C.c_int), ("outflow", C.c_int), ("mem", C.c_int),
        ("tau", C.c_double), ("tau_bulk", C.c_double), ("lambda_trt", C.c_double), ("cs_smag", C.c_double),
        ("g", C.c_double * 3), ("u_in", C.c_double * 3), ("rho_out", C.c_double), ("u_wall", C.c_double * 3),
        ("center", C.c_double * 3), ("r_max", C.c_double), ("s3", C.c_double), ("s4", C.c_double),
        ("thermal", C.c_int), ("tau_t", C.c_double), ("t_ref", C.c_double), ("beta_g", C.c_double),
        ("t_south", C.c_double), ("t_north", C.c_double),
    ]


_lib = None
_ref = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists() or ORACLE_SO.stat().st_mtime < (HERE / "wake_oracle.cpp").stat().st_mtime:
            build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        vp, I, D = C.c_void_p, C.c_int, C.c_double
        sig = {
            "og_create": (vp, [I, I, I, I, I]), "og_destroy": (None, [vp]),
            "og_set_params": (None, [vp, C.POINTER(Params)]), "og_set_cell_types": (None, [vp, vp]),
            "og_set_state": (None, [vp, vp, vp, vp, vp, vp]), "og_set_links": (None, [vp, I, vp, vp, vp, vp]),
            "og_step": (None, [vp, I, vp]), "og_get_f": (None, [vp, vp]),
            "og_get_macro": (None, [vp, vp, vp, vp, vp, vp]), "og_forces": (None, [vp, vp]),
            "og_equilibrium": (None, [I, I, C.c_longlong, vp, vp, vp, vp, vp]),
            "og_collide_nodes": (None, [vp, C.c_longlong, vp, vp, vp, vp, vp, vp, vp]),
            "og_d3q19_minv": (D, [I, I, I]), "og_strouhal_frequency": (D, [vp, I, D]),
            "og_smagorinsky_tau": (D, [I, vp, D, D, D, D, D, D]),
            "og_set_thermal_state": (None, [vp, vp]), "og_get_temperature": (None, [vp, vp]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def ref() -> C.CDLL | None:
    """The reference library, or None where it was never built."""
    global _ref
    if _ref is None:
        if not REF_SO.exists():
            try:
                build_reference()
            except Exception:
                return None
        if not REF_SO.exists():
            return None
        L = C.CDLL(str(REF_SO))
        vp, I, F = C.c_void_p, C.c_int, C.c_float
        sig = {
            "ref2d_create": (vp, [I, I, F]), "ref2d_destroy": (None, [vp]),
            "ref2d_init_fields": (None, [vp, vp, vp, vp]), "ref2d_set_cell_type": (None, [vp, I, I, I]),
            "ref2d_set_solid_circle": (None, [vp, F, F, F]), "ref2d_set_inflow_west": (None, [vp, F, F]),
            "ref2d_set_outflow_east": (None, [vp, F]), "ref2d_set_moving_wall_north": (None, [vp, F]),
            "ref2d_step": (None, [vp, I, F, F, I, F, I]),
            "ref2d_step_forces": (None, [vp, I, F, F, I, F, I, F, F, F, vp]),
            "ref2d_get_f": (None, [vp, vp]), "ref2d_get_macro": (None, [vp, vp, vp, vp, vp]),
            "ref2d_get_cell_types": (None, [vp, vp]), "ref2d_total_mass": (F, [vp]),
            "ref2d_total_ke": (F, [vp]), "ref2d_max_speed": (F, [vp]),
            "ref3d_create": (vp, [I, I, I, F]), "ref3d_destroy": (None, [vp]),
            "ref3d_init_fields": (None, [vp, vp, vp, vp, vp]), "ref3d_set_periodic": (None, [vp, I]),
            "ref3d_set_cell_type": (None, [vp, I, I, I, I]), "ref3d_set_solid_sphere": (None, [vp, F, F, F, F]),
            "ref3d_build_curved_sphere_links": (None, [vp, F, F, F, F]),
            "ref3d_set_moving_wall_top": (None, [vp, F, F]),
            "ref3d_step": (None, [vp, I, F, F, F, I, F, I]),
            "ref3d_step_forces": (None, [vp, I, F, F, F, I, F, I, F, F, F, F, vp]),
            "ref3d_get_f": (None, [vp, vp]), "ref3d_get_macro": (None, [vp, vp, vp, vp, vp, vp]),
            "ref3d_get_cell_types": (None, [vp, vp]), "ref3d_num_links": (I, [vp]),
            "ref3d_get_links": (None, [vp, vp, vp, vp]), "ref3d_is_periodic": (I, [vp]),
            "ref3d_total_mass": (F, [vp]), "ref3d_total_ke": (F, [vp]), "ref3d_max_speed": (F, [vp]),
            "ref_strouhal_frequency": (F, [vp, I, F]),
            "ref_vtk_export_2d": (I, [vp, C.c_char_p, vp]), "ref_vtk_export_3d": (I, [vp, C.c_char_p, vp, vp]),
            "ref_vtk_pvd": (I, [C.c_char_p, C.c_char_p, I, I, I, F]),
            "compute_vorticity_2d": (None, [vp, vp, vp, I, I]),
            "compute_vorticity_and_q_criterion_3d": (None, [vp, vp, vp, vp, vp, vp, vp, I, I, I]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _ref = L
    return _ref


class OracleGrid:
    """CPU oracle lattice (float or double) following the reference step order."""

    def __init__(self, q: int, nx: int, ny: int, nz: int = 1, prec: int = 64):
        self.q, self.nx, self.ny, self.nz, self.prec = q, nx, ny, nz, prec
        self.n = nx * ny * nz
        self._h = lib().og_create(q, nx, ny, nz, prec)
        self.params = Params()
        self.params.collision = 2
        self.params.tau = 0.6
        self.params.tau_bulk = 1.63 if q == 9 else (1.19 if q == 19 else 1.0)
        self.params.lambda_trt = 0.25
        self.params.cs_smag = 0.14
        self.params.rho_out = 1.0
        self.params.s3 = 1.0
        self.params.s4 = 1.0

    def __del__(self):
        if getattr(self, "_h", None):
            lib().og_destroy(self._h)
            self._h = None

    def configure(self, **kw):
        for k, v in kw.items():
            if k in ("g", "u_in", "u_wall", "center"):
                arr = getattr(self.params, k)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(self.params, k, v)
        lib().og_set_params(self._h, C.byref(self.params))

    def set_cell_types(self, t):
        t = np.ascontiguousarray(t, np.uint8).ravel()
        lib().og_set_cell_types(self._h, _addr(t))

    def set_state(self, f, rho=None, ux=None, uy=None, uz=None):
        f = np.ascontiguousarray(f, np.float64).reshape(self.q, self.n)
        n = self.n
        z = np.zeros(n)
        rho = np.ascontiguousarray(rho if rho is not None else f.sum(0), np.float64)
        ux = np.ascontiguousarray(ux if ux is not None else z, np.float64)
        uy = np.ascontiguousarray(uy if uy is not None else z, np.float64)
        uz = np.ascontiguousarray(uz if uz is not None else z, np.float64)
        lib().og_set_state(self._h, _addr(f), _addr(rho), _addr(ux), _addr(uy), _addr(uz))

    def set_thermal_state(self, t5):
        """D2Q5 temperature populations [5][n] (D2Q9 grids configured with thermal=1)."""
        t5 = np.ascontiguousarray(t5, np.float64).reshape(5, self.n)
        lib().og_set_thermal_state(self._h, _addr(t5))

    def temperature(self):
        out = np.empty(self.n)
        lib().og_get_temperature(self._h, _addr(out))
        return out

    def set_links(self, idx, q, delta, uw=None):
        idx = np.ascontiguousarray(idx, np.int32)
        q = np.ascontiguousarray(q, np.int32)
        delta = np.ascontiguousarray(delta, np.float64)
        uw = None if uw is None else np.ascontiguousarray(uw, np.float64)
        lib().og_set_links(self._h, len(idx), _addr(idx), _addr(q), _addr(delta), _addr(uw))

    def step(self, n: int = 1, forces: bool = False):
        hist = np.zeros((n, 3)) if forces else None
        lib().og_step(self._h, n, _addr(hist))
        return hist

    def f(self):
        out = np.empty((self.q, self.n))
        lib().og_get_f(self._h, _addr(out))
        return out

    def macro(self):
        out = {k: np.empty(self.n) for k in ("rho", "ux", "uy", "uz", "speed")}
        lib().og_get_macro(self._h, *[_addr(out[k]) for k in ("rho", "ux", "uy", "uz", "speed")])
        return out

    def forces(self):
        out = np.empty(3)
        lib().og_forces(self._h, _addr(out))
        return out


def equilibrium(q: int, rho, ux, uy, uz=None, prec: int = 32) -> np.ndarray:
    rho = np.ascontiguousarray(rho, np.float64).ravel()
    ux = np.ascontiguousarray(ux, np.float64).ravel()
    uy = np.ascontiguousarray(uy, np.float64).ravel()
    uz = None if uz is None else np.ascontiguousarray(uz, np.float64).ravel()
    f = np.empty((q, len(rho)))
    lib().og_equilibrium(q, prec, len(rho), _addr(rho), _addr(ux), _addr(uy), _addr(uz), _addr(f))
    return f


def strouhal_frequency(signal, dt=1.0) -> float:
    s = np.ascontiguousarray(signal, np.float64)
    return float(lib().og_strouhal_frequency(_addr(s), len(s), dt))


def vorticity_2d(ux, uy, nx: int, ny: int, dtype=np.float32) -> np.ndarray:
    """omega_z = 0.5 (uy[x+1] - uy[x-1]) - 0.5 (ux[y+1] - ux[y-1]), periodic wrap
    (src/ispc/analytics_kernels.ispc:4-29). Each operation rounds to `dtype`, in the
    reference's order (float32: the reference expression evaluated without contraction)."""
    t = np.dtype(dtype).type
    ux = np.asarray(ux, dtype).reshape(ny, nx)
    uy = np.asarray(uy, dtype).reshape(ny, nx)
    h = t(0.5)
    duy_dx = h * (np.roll(uy, -1, axis=1) - np.roll(uy, 1, axis=1))
    dux_dy = h * (np.roll(ux, -1, axis=0) - np.roll(ux, 1, axis=0))
    return (duy_dx - dux_dy).ravel()


def vorticity_q_3d(ux, uy, uz, nx: int, ny: int, nz: int, dtype=np.float32):
    """Vorticity vector and Q = 0.5 (|Omega|^2 - |S|^2) by central differences with
    periodic wrap (src/ispc/analytics_kernels.ispc:31-110), every operation rounded
    to `dtype` in the reference's order. Returns (omega_x, omega_y, omega_z, Q)."""
    t = np.dtype(dtype).type
    u = [np.asarray(a, dtype).reshape(nz, ny, nx) for a in (ux, uy, uz)]
    h, two = t(0.5), t(2.0)

    def d(a, axis):  # axis 2 = x, 1 = y, 0 = z
        return h * (np.roll(a, -1, axis=axis) - np.roll(a, 1, axis=axis))

    dux_dx, dux_dy, dux_dz = d(u[0], 2), d(u[0], 1), d(u[0], 0)
    duy_dx, duy_dy, duy_dz = d(u[1], 2), d(u[1], 1), d(u[1], 0)
    duz_dx, duz_dy, duz_dz = d(u[2], 2), d(u[2], 1), d(u[2], 0)
    wx, wy, wz = duz_dy - duy_dz, dux_dz - duz_dx, duy_dx - dux_dy
    s_xy, s_yz, s_xz = h * (dux_dy + duy_dx), h * (duy_dz + duz_dy), h * (dux_dz + duz_dx)
    norm_s = ((dux_dx * dux_dx + duy_dy * duy_dy) + duz_dz * duz_dz) + two * ((s_xy * s_xy + s_yz * s_yz) + s_xz * s_xz)
    o_xy, o_yz, o_xz = h * (dux_dy - duy_dx), h * (duy_dz - duz_dy), h * (dux_dz - duz_dx)
    norm_o = two * ((o_xy * o_xy + o_yz * o_yz) + o_xz * o_xz)
    q = h * (norm_o - norm_s)
    return wx.ravel(), wy.ravel(), wz.ravel(), q.ravel()


def d3q19_minv(rounded: bool) -> np.ndarray:
    return np.array([[lib().og_d3q19_minv(int(rounded), q, k) for k in range(19)] for q in range(19)])


# ----------------------------------------------------------------------------- reference grids
class RefGrid2D:
    """wake::LatticeGrid2D from the reference's own sources (oracle/_ref)."""

    def __init__(self, nx, ny, tau):
        self.L = ref()
        if self.L is None:
            raise RuntimeError("reference library not built")
        self.nx, self.ny, self.n = nx, ny, nx * ny
        self._h = self.L.ref2d_create(nx, ny, tau)

    def __del__(self):
        if getattr(self, "_h", None):
            self.L.ref2d_destroy(self._h)
            self._h = None

    def init_fields(self, rho, ux, uy):
        a = [np.ascontiguousarray(v, np.float32).ravel() for v in (rho, ux, uy)]
        self.L.ref2d_init_fields(self._h, *[_addr(v) for v in a])

    def f(self):
        out = np.empty((9, self.n), np.float32)
        self.L.ref2d_get_f(self._h, _addr(out))
        return out

    def macro(self):
        out = {k: np.empty(self.n, np.float32) for k in ("rho", "ux", "uy", "speed")}
        self.L.ref2d_get_macro(self._h, *[_addr(out[k]) for k in ("rho", "ux", "uy", "speed")])
        return out

    def cell_types(self):
        out = np.empty(self.n, np.uint8)
        self.L.ref2d_get_cell_types(self._h, _addr(out))
        return out

    def step(self, n, collision, gx=0.0, gy=0.0, use_les=False, cs=0.14):
        self.L.ref2d_step(self._h, collision, gx, gy, int(use_les), cs, n)

    def step_forces(self, n, collision, cx, cy, r_max, gx=0.0, gy=0.0, use_les=False, cs=0.14):
        hist = np.zeros((n, 3), np.float32)
        self.L.ref2d_step_forces(self._h, collision, gx, gy, int(use_les), cs, n, cx, cy, r_max, _addr(hist))
        return hist


class RefGrid3D:
    """wake::LatticeGrid3D from the reference's own sources (oracle/_ref)."""

    def __init__(self, nx, ny, nz, tau):
        self.L = ref()
        if self.L is None:
            raise RuntimeError("reference library not built")
        self.nx, self.ny, self.nz, self.n = nx, ny, nz, nx * ny * nz
        self._h = self.L.ref3d_create(nx, ny, nz, tau)

    def __del__(self):
        if getattr(self, "_h", None):
            self.L.ref3d_destroy(self._h)
            self._h = None

    def init_fields(self, rho, ux, uy, uz):
        a = [np.ascontiguousarray(v, np.float32).ravel() for v in (rho, ux, uy, uz)]
        self.L.ref3d_init_fields(self._h, *[_addr(v) for v in a])

    def f(self):
        out = np.empty((19, self.n), np.float32)
        self.L.ref3d_get_f(self._h, _addr(out))
        return out

    def macro(self):
        out = {k: np.empty(self.n, np.float32) for k in ("rho", "ux", "uy", "uz", "speed")}
        self.L.ref3d_get_macro(self._h, *[_addr(out[k]) for k in ("rho", "ux", "uy", "uz", "speed")])
        return out

    def cell_types(self):
        out = np.empty(self.n, np.uint8)
        self.L.ref3d_get_cell_types(self._h, _addr(out))
        return out

    def links(self):
        n = self.L.ref3d_num_links(self._h)
        idx, q, d = np.empty(n, np.int32), np.empty(n, np.int32), np.empty(n, np.float32)
        self.L.ref3d_get_links(self._h, _addr(idx), _addr(q), _addr(d))
        return idx, q, d

    def step(self, n, collision, g=(0.0, 0.0, 0.0), use_les=False, cs=0.14):
        self.L.ref3d_step(self._h, collision, *g, int(use_les), cs, n)

    def step_forces(self, n, collision, center, r_max, g=(0.0, 0.0, 0.0), use_les=False, cs=0.14):
        hist = np.zeros((n, 3), np.float32)
        self.L.ref3d_step_forces(self._h, collision, *g, int(use_les), cs, n, *center, r_max, _addr(hist))
        return hist
