"""ctypes binding of libwake_b200.so (C ABI in include/wake_gpu.h).

The library is built in-tree (``python wake_b200/build.py``, ``make -C
wake_b200/csrc`` or ``__graft_entry__.build()``). Importing this module without it raises
ImportError: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("WAKE_B200_LIB", _HERE / "libwake_b200.so"))

if not LIB_PATH.exists():
    raise ImportError(f"wake_b200: {LIB_PATH} is missing; build it with `python wake_b200/build.py`")

lib = C.CDLL(str(LIB_PATH))

fp = C.POINTER(C.c_float)
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p
F, I, D, LL = C.c_float, C.c_int, C.c_double, C.c_longlong

# Every pointer argument is declared as void* so numpy arrays (host) and torch
# CUDA tensors (device) can both be passed by address.
_PROTOS = {
    # errors
    "wake_gpu_last_error": (C.c_char_p, []),
    "wake_gpu_last_error_code": (I, []),
    "wake_gpu_clear_error": (None, []),
    "wake_gpu_version": (C.c_char_p, []),
    "wake_gpu_cache_trim": (LL, []),
    "wake_gpu_cache_bytes": (LL, []),
    # drop-in kernels (ISPC signatures)
    "d2q9_collide_bgk": (None, [vp, vp, vp, vp, vp, vp, F, F, F, I]),
    "d2q9_collide_trt": (None, [vp, vp, vp, vp, vp, vp, F, F, F, F, I]),
    "d2q9_collide_mrt": (None, [vp, vp, vp, vp, vp, vp, F, F, F, F, I]),
    "d2q9_stream_periodic": (None, [vp, vp, I, I]),
    "d2q9_stream_with_boundaries": (None, [vp, vp, vp, I, I, F, F]),
    "d2q9_apply_bounce_back": (None, [vp, vp, F, F, I]),
    "d2q9_apply_zou_he_inflow_west": (None, [vp, vp, vp, vp, F, F, I, I]),
    "d2q9_apply_zou_he_outflow_east": (None, [vp, vp, vp, vp, F, I, I]),
    "d2q9_apply_convective_outflow_east": (None, [vp, vp, F, I, I]),
    "d2q9_compute_smagorinsky_tau": (None, [vp, vp, vp, vp, vp, F, F, I]),
    "d2q9_compute_macroscopic_moments": (None, [vp, vp, vp, vp, I]),
    "d2q9_compute_macroscopic_moments_forced": (None, [vp, vp, vp, vp, F, F, I]),
    "d2q9_compute_velocity_magnitude": (None, [vp, vp, vp, I]),
    "d2q9_compute_momentum_exchange_forces": (None, [vp, vp, I, I, F, F, F, vp, vp, vp]),
    "d3q19_collide_bgk": (None, [vp, vp, vp, vp, vp, vp, vp, F, F, F, F, I]),
    "d3q19_collide_trt": (None, [vp, vp, vp, vp, vp, vp, vp, F, F, F, F, F, I]),
    "d3q19_collide_mrt": (None, [vp, vp, vp, vp, vp, vp, vp, F, F, F, F, F, I]),
    "d3q19_stream_periodic": (None, [vp, vp, I, I, I]),
    "d3q19_stream_with_boundaries": (None, [vp, vp, vp, I, I, I, F, F, F]),
    "d3q19_apply_curved_bfl": (None, [vp, vp, vp, vp, vp, vp, vp, vp, I, I, I, I]),
    "d3q19_compute_smagorinsky_tau": (None, [vp, vp, vp, vp, vp, vp, F, F, I]),
    "d3q19_compute_macroscopic_moments": (None, [vp, vp, vp, vp, vp, I]),
    "d3q19_compute_macroscopic_moments_forced": (None, [vp, vp, vp, vp, vp, F, F, F, I]),
    "d3q19_compute_velocity_magnitude": (None, [vp, vp, vp, vp, I]),
    "d3q19_compute_momentum_exchange_forces": (None, [vp, vp, I, I, I, F, F, F, F, vp, vp, vp]),
    "d3q27_collide": (None, [vp, vp, vp, vp, vp, vp, vp, F, F, F, F, F, I]),
    "d3q27_compute_macroscopic_moments": (None, [vp, vp, vp, vp, vp, I]),
    "d3q27_stream_periodic": (None, [vp, vp, I, I, I]),
    "thermal_collide_d2q9": (None, [vp, vp, vp, vp, vp, vp, F, I]),
    "thermal_compute_buoyancy_force_2d": (None, [vp, vp, F, F, F, I]),
    "thermal_apply_isothermal_wall": (None, [vp, I, I, I, F]),
    "ibm_interpolate_velocity_2d": (None, [vp, vp, vp, vp, vp, vp, I, I, I]),
    "ibm_spread_force_2d": (None, [vp, vp, vp, vp, vp, vp, vp, I, I, I]),
    "compute_vorticity_2d": (None, [vp, vp, vp, I, I]),
    "compute_vorticity_and_q_criterion_3d": (None, [vp, vp, vp, vp, vp, vp, vp, I, I, I]),
    # fused engine
    "wake_grid_create": (vp, [I, I, I, I, F, I]),
    "wake_grid_destroy": (None, [vp]),
    "wake_grid_set_stream": (I, [vp, vp]),
    "wake_grid_set_model": (I, [vp, I, I, F, F, F, I, F, F]),
    "wake_grid_set_relaxation_time": (I, [vp, F]),
    "wake_grid_set_cell_type": (I, [vp, I, I, I, I]),
    "wake_grid_set_cell_types": (I, [vp, vp]),
    "wake_grid_get_cell_types": (I, [vp, vp]),
    "wake_grid_set_solid_box": (I, [vp, I, I, I, I, I, I]),
    "wake_grid_set_solid_circle": (I, [vp, F, F, F]),
    "wake_grid_set_solid_sphere": (I, [vp, F, F, F, F]),
    "wake_grid_set_inflow_west": (I, [vp, F, F, F]),
    "wake_grid_set_outflow_east": (I, [vp, F]),
    "wake_grid_set_moving_wall": (I, [vp, F, F, F]),
    "wake_grid_set_periodic": (I, [vp, I, I]),
    "wake_grid_set_curved_links": (I, [vp, I, vp, vp, vp, vp, vp, vp]),
    "wake_grid_build_curved_sphere_links": (I, [vp, F, F, F, F]),
    "wake_grid_num_curved_links": (I, [vp]),
    "wake_grid_get_curved_links": (I, [vp, vp, vp, vp]),
    "wake_grid_initialize": (I, [vp, F, F, F, F]),
    "wake_grid_initialize_fields": (I, [vp, vp, vp, vp, vp]),
    "wake_grid_initialize_noise": (I, [vp, F, F, F, F, F, C.c_ulonglong, LL]),
    "wake_grid_set_populations": (I, [vp, vp]),
    "wake_grid_set_populations_device": (I, [vp, vp]),
    "wake_grid_enable_forces": (I, [vp, F, F, F, F, I]),
    "wake_grid_disable_forces": (I, [vp]),
    "wake_grid_get_force_history": (I, [vp, vp, I]),
    "wake_grid_force_count": (LL, [vp]),
    "wake_grid_step": (I, [vp, I, F, F, F]),
    "wake_grid_use_graph": (I, [vp, I]),
    "wake_grid_prepare_steps": (I, [vp, F, F, F]),
    "wake_grid_step_count": (LL, [vp]),
    "wake_grid_synchronize": (I, [vp]),
    "wake_grid_get_populations": (I, [vp, vp]),
    "wake_grid_get_macroscopic": (I, [vp, vp, vp, vp, vp, vp]),
    "wake_grid_diagnostics": (I, [vp, vp, vp, vp]),
    "wake_grid_total_mass": (I, [vp, vp]),
    "wake_grid_info": (I, [vp, vp, vp, vp, vp, vp, vp]),
    "wake_grid_state_buffer": (vp, [vp, I]),
    "wake_grid_set_block": (I, [vp, I]),
    "wake_grid_get_block": (I, [vp]),
    "wake_grid_launches_per_step": (I, [vp]),
    "wake_grid_set_kernel": (I, [vp, I]),
    "wake_grid_get_kernel": (I, [vp]),
    "wake_batch_set_kernel": (I, [vp, I]),
    "wake_grid_time_bulk_launches": (I, [vp, I]),
    "wake_grid_bulk_launch_times": (I, [vp, vp, vp, vp]),
    "wake_grid_set_solid_ellipse": (I, [vp, F, F, F, F, F]),
    "wake_grid_enable_thermal": (I, [vp, F, F, F, F, F]),
    "wake_grid_initialize_temperature": (I, [vp, vp]),
    "wake_grid_get_temperature": (I, [vp, vp]),
    "wake_grid_device_bytes": (LL, [vp]),
    "wake_grid_estimate_bytes": (LL, [I, I, I, I, I, I]),
    "wake_grid_release_scratch": (I, [vp]),
    "wake_batch_create": (vp, [I, I]),
    "wake_batch_destroy": (None, [vp]),
    "wake_batch_add": (I, [vp, vp]),
    "wake_batch_remove": (I, [vp, vp]),
    "wake_batch_size": (I, [vp]),
    "wake_batch_set_stream": (I, [vp, vp]),
    "wake_batch_use_graph": (I, [vp, I]),
    "wake_batch_set_block": (I, [vp, I, I]),
    "wake_batch_get_block": (I, [vp]),
    "wake_batch_step": (I, [vp, I]),
    "wake_batch_synchronize": (I, [vp]),
    "wake_batch_info": (I, [vp, vp, vp, vp, vp]),
    "wake_batch_autotune": (I, [vp, I, vp]),
    "wake_batch_host_seconds": (I, [vp, vp, vp, vp]),
    "wake_grid_compute_vorticity": (I, [vp, vp]),
    "wake_grid_compute_3d_features": (I, [vp, vp, vp, vp, vp]),
    "wake_grid_max_vorticity": (I, [vp, vp]),
    "wake_field_abs_max": (I, [vp, LL, vp]),
    "wake_vtk_write_vti_2d": (I, [C.c_char_p, I, I, vp, vp, vp, vp, vp, vp, I]),
    "wake_vtk_write_vti_3d": (I, [C.c_char_p, I, I, I, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, I]),
    "wake_vtk_write_pvd": (I, [C.c_char_p, C.c_char_p, I, I, I, F]),
    "wake_grid_export_vti": (I, [vp, C.c_char_p, I, I]),
    "wake_telemetry_create": (vp, []),
    "wake_telemetry_destroy": (None, [vp]),
    "wake_telemetry_clear": (None, [vp]),
    "wake_telemetry_record_aero": (I, [vp, C.c_ulonglong, F, F, F, F, F, F, F, F, F]),
    "wake_telemetry_record_history": (I, [vp, vp, I, LL, I, I, F, F, F, F]),
    "wake_telemetry_record_performance": (I, [vp, C.c_ulonglong, D, D, F, F, F]),
    "wake_telemetry_count": (I, [vp, I]),
    "wake_telemetry_get_coefficients": (I, [vp, I, vp]),
    "wake_telemetry_write_aero_csv": (I, [vp, C.c_char_p]),
    "wake_telemetry_write_performance_csv": (I, [vp, C.c_char_p]),
    "wake_telemetry_write_summary_json": (I, [vp, C.c_char_p, C.c_char_p, F, F]),
    "wake_strouhal_frequency": (D, [vp, I, D]),
}

for _name, (_res, _args) in _PROTOS.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args

EXPORTED = tuple(_PROTOS)


class WakeError(RuntimeError):
    """Error reported by the library (message from wake_gpu_last_error)."""


def check(rc: int) -> int:
    if rc < 0:
        msg = lib.wake_gpu_last_error().decode(errors="replace")
        lib.wake_gpu_clear_error()
        raise WakeError(f"wake_b200 error {rc}: {msg}")
    return rc


def addr(a) -> int | None:
    """Address of a numpy array (host) or torch tensor (device or host)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
