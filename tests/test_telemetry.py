"""Telemetry files: the library's writers against the reference's own TelemetryExporter.

The reference exporter (src/export/csv_telemetry.cpp, compiled from its sources
into oracle/_ref) writes the same records; the files must be identical bytes.
Host code only: no GPU needed (the reference build exists where its sources do).
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from wake_b200.telemetry import TelemetryExporter

REF = oracle.ref()
pytestmark = pytest.mark.skipif(REF is None, reason="reference build oracle/_ref is absent")


def _ref_exporter():
    L = REF
    vp, F, D, ULL = C.c_void_p, C.c_float, C.c_double, C.c_ulonglong
    L.ref_telemetry_create.restype = vp
    L.ref_telemetry_destroy.argtypes = [vp]
    L.ref_telemetry_record_aero.argtypes = [vp, ULL, F, F, F, F, F, F, F, F, F]
    L.ref_telemetry_record_performance.argtypes = [vp, ULL, D, D, F, F, F]
    L.ref_telemetry_write.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p, F, F]
    L.ref_telemetry_write.restype = C.c_int
    return L


def _history(n, seed, is3d):
    rng = np.random.default_rng(seed)
    h = np.empty((n, 3))
    h[:, 0] = 0.02 + 1e-3 * rng.standard_normal(n)
    h[:, 1] = 5e-3 * np.sin(np.arange(n) * 0.05) + 1e-4 * rng.standard_normal(n)
    h[:, 2] = (1e-4 if is3d else 3e-2) * rng.standard_normal(n)
    return h


@pytest.mark.parametrize("is3d", [False, True])
def test_files_match_reference_exporter(tmp_path, is3d):
    L = _ref_exporter()
    n, first, every = 997, 1, 10
    rho, u, area, chord = 1.0, 0.05, (452.389 if is3d else 20.0), 20.0
    hist = _history(n, 7 + int(is3d), is3d)
    ours = TelemetryExporter()
    ours.record_history(hist, first_step=first, every=every, is3d=is3d, rho_inf=rho, u_inf=u, area=area, chord=chord)
    ref = L.ref_telemetry_create()
    for i in range(n):
        step = first + i
        if step % every:
            continue
        fx, fy, c = (float(np.float32(v)) for v in hist[i])
        fz, tz = (c, 0.0) if is3d else (0.0, c)
        L.ref_telemetry_record_aero(ref, step, float(np.float32(step)), fx, fy, fz, tz, rho, u, area, chord)
    rng = np.random.default_rng(3)
    for k in range(40):
        vals = (k * 20, float(rng.uniform(0.1, 3.0)), float(rng.uniform(1e3, 4e4)), float(rng.uniform(0, 0.1)),
                float(rng.uniform(6e4, 7e4)), float(rng.uniform(0, 2.0)))
        ours.record_performance(*vals)
        L.ref_telemetry_record_performance(ref, *vals)
    assert ours.aero_count() == len([s for s in range(first, first + n) if s % every == 0])
    for which, fn in ((0, "aero.csv"), (1, "perf.csv"), (2, "summary.json")):
        a, b = tmp_path / f"ours_{fn}", tmp_path / f"ref_{fn}"
        if which == 0:
            ours.write_aero_csv(a)
        elif which == 1:
            ours.write_performance_csv(a)
        else:
            ours.write_summary_json(a, "karman_vortex", 0.1953125, 0.00048828125)
        assert L.ref_telemetry_write(ref, which, str(b).encode(), b"karman_vortex", 0.1953125, 0.00048828125) == 0
        assert a.read_bytes() == b.read_bytes(), fn
    L.ref_telemetry_destroy(ref)
    ours.close()


def test_empty_exporter_matches_reference(tmp_path):
    L = _ref_exporter()
    ours, ref = TelemetryExporter(), L.ref_telemetry_create()
    ours.write_summary_json(tmp_path / "a.json", "empty")
    L.ref_telemetry_write(ref, 2, str(tmp_path / "b.json").encode(), b"empty", 0.0, 0.0)
    assert (tmp_path / "a.json").read_bytes() == (tmp_path / "b.json").read_bytes()
    L.ref_telemetry_destroy(ref)
