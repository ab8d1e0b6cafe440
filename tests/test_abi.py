"""The C-ABI library loads and exports every function include/wake_gpu.h declares (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def header_functions():
    text = (ROOT / "include" / "wake_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;]*\)\s*;", text, flags=re.M)
    return sorted(set(names))


def test_header_has_all_reference_kernels():
    names = set(header_functions())
    # all 35 ISPC exports of the reference (src/ispc/*.ispc): the library links in place of it
    ispc = {
        "d2q9_collide_bgk", "d2q9_collide_trt", "d2q9_collide_mrt", "d2q9_stream_periodic",
        "d2q9_stream_with_boundaries", "d2q9_apply_bounce_back", "d2q9_apply_zou_he_inflow_west",
        "d2q9_apply_zou_he_outflow_east", "d2q9_apply_convective_outflow_east", "d2q9_compute_smagorinsky_tau",
        "d2q9_compute_macroscopic_moments", "d2q9_compute_macroscopic_moments_forced",
        "d2q9_compute_velocity_magnitude", "d2q9_compute_momentum_exchange_forces", "d3q19_collide_bgk",
        "d3q19_collide_trt", "d3q19_collide_mrt", "d3q19_stream_periodic", "d3q19_stream_with_boundaries",
        "d3q19_apply_curved_bfl", "d3q19_compute_smagorinsky_tau", "d3q19_compute_macroscopic_moments",
        "d3q19_compute_macroscopic_moments_forced", "d3q19_compute_velocity_magnitude",
        "d3q19_compute_momentum_exchange_forces", "d3q27_collide", "d3q27_compute_macroscopic_moments",
        "d3q27_stream_periodic", "thermal_collide_d2q9", "thermal_compute_buoyancy_force_2d",
        "thermal_apply_isothermal_wall", "compute_vorticity_2d", "compute_vorticity_and_q_criterion_3d",
        "ibm_interpolate_velocity_2d", "ibm_spread_force_2d",
    }
    assert ispc <= names


def test_library_exports_every_declared_symbol():
    import wake_b200 as wb

    lib = C.CDLL(str(wb.LIB_PATH))
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(wb.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(header_functions()) <= exported
    # every binding the Python package declares is a header function
    assert set(wb.EXPORTED) <= set(header_functions())


def test_error_channel_and_version():
    import wake_b200 as wb

    assert wb.lib.wake_gpu_version().startswith(b"wake_b200")
    wb.lib.wake_gpu_clear_error()
    assert wb.lib.wake_gpu_last_error() == b""
    # invalid arguments are rejected before any device work
    assert not wb.lib.wake_grid_create(10, 8, 8, 1, 0.6, 0)
    assert wb.lib.wake_gpu_last_error_code() == -1
    assert not wb.lib.wake_grid_create(9, 8, 8, 2, 0.6, 0)
    assert not wb.lib.wake_grid_create(19, 8, 8, 8, 0.5, 0)
    assert wb.lib.wake_grid_step(None, 1, 0.0, 0.0, 0.0) == -1
    wb.lib.wake_gpu_clear_error()


def test_strouhal_fp64_matches_reference_kat(golden):
    """FFT peak of tests/unit/test_forces_momentum_exchange.cpp:71-91 (host code, FP64)."""
    import wake_b200 as wb

    d = golden("kat")
    f = wb.strouhal_frequency(d["strouhal_signal"], 1.0)
    assert abs(f - 0.025) <= 0.003
    assert abs(f - float(d["strouhal_freq"])) <= 1e-6


def test_strouhal_uses_first_4096_samples():
    import wake_b200 as wb

    t = np.arange(6000)
    s = np.where(t < 4096, np.sin(2 * np.pi * 0.05 * t), np.sin(2 * np.pi * 0.2 * t))
    assert abs(wb.strouhal_frequency(s) - 0.05) < 1e-3
