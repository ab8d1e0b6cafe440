"""Drop-in kernel entry points (reference ISPC signatures) vs the reference's outputs.

The golden file percall.npz holds inputs and outputs of single calls of the
reference's own kernels. Each entry point runs twice: with host pointers
(numpy; staged through the device) and with device pointers (torch CUDA
tensors; used in place). Arithmetic kernels must agree to 2e-6 relative
(FP32 with a different operation order).

Streaming moves values unchanged, except that pulls from a moving-wall node add
the wall term 2 w_q 3 (c_q . u_w); the reference's build folds that product under
fast-math, so those entries may differ in the last bit (STREAM_ULP).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

wb = pytest.importorskip("wake_b200")
torch = pytest.importorskip("torch")

ARITH_TOL = 2e-6
STREAM_ULP = 6e-8  # two units in the last place at |f| < 0.5


def same_stream(a, b):
    return np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max() <= STREAM_ULP


@pytest.fixture(params=["host", "device"])
def mode(request):
    return request.param


class Args:
    """Holds call buffers as numpy (host) or torch CUDA tensors (device)."""

    def __init__(self, mode):
        self.mode = mode
        self.bufs = []

    def __call__(self, arr):
        arr = np.ascontiguousarray(arr)
        if self.mode == "host":
            b = arr.copy()
        else:
            b = torch.from_numpy(arr.copy()).cuda()
        self.bufs.append(b)
        return b

    @staticmethod
    def ptr(b):
        return b.data_ptr() if hasattr(b, "data_ptr") else b.ctypes.data

    @staticmethod
    def np(b):
        return b.cpu().numpy() if hasattr(b, "cpu") else b


def close(a, b, tol=ARITH_TOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return np.abs(a - b).max() <= tol * scale


@pytest.mark.parametrize("pref,name,taus", [
    ("d2q9", "bgk", (0.7,)), ("d2q9", "trt", (0.7, 1.2)), ("d2q9", "mrt", (0.7, 1.6)),
    ("d3q19", "bgk", (0.75,)), ("d3q19", "trt", (0.75, 1.3)), ("d3q19", "mrt", (0.75, 1.2)),
    ("d3q27", "collide", (0.75, 1.3)),
])
def test_collide(golden, mode, pref, name, taus):
    d = golden("percall")
    A = Args(mode)
    f = A(d[f"{pref}_f"])
    Q, count = d[f"{pref}_f"].shape
    out = A(np.zeros_like(d[f"{pref}_f"]))
    ct = A(d[f"{pref}_ct"])
    mom = [A(np.zeros(count, np.float32)) for _ in range(3 if Q == 9 else 4)]
    fn = getattr(wb.lib, "d3q27_collide" if pref == "d3q27" else f"{pref}_collide_{name}")
    g = (1e-5, -2e-5) if Q == 9 else (1e-5, -2e-5, 3e-5)
    fn(A.ptr(f), A.ptr(out), A.ptr(ct), *[A.ptr(m) for m in mom], *taus, *g, count)
    key = f"{pref}_{name}"
    assert close(A.np(out), d[f"{key}_out"])
    assert close(A.np(mom[0]), d[f"{key}_rho"])
    for i, k in enumerate(("ux", "uy", "uz")[: len(mom) - 1]):
        assert close(A.np(mom[i + 1]), d[f"{key}_{k}"], 1e-5)
    # solid nodes are copied through unchanged (tests/unit/test_d2q9_collision.cpp:124-131)
    solid = d[f"{pref}_ct"] == 1
    assert np.array_equal(A.np(out)[:, solid], d[f"{pref}_f"][:, solid])


def test_stream_2d(golden, mode):
    d = golden("percall")
    A = Args(mode)
    f, ct = A(d["s2_f"]), A(d["s2_ct"])
    out = A(np.zeros_like(d["s2_f"]))
    wb.lib.d2q9_stream_with_boundaries(A.ptr(f), A.ptr(out), A.ptr(ct), 20, 12, 0.08, 0.0)
    assert same_stream(A.np(out), d["s2_stream"])
    per = A(np.zeros_like(d["s2_f"]))
    wb.lib.d2q9_stream_periodic(A.ptr(f), A.ptr(per), 20, 12)
    assert same_stream(A.np(per), d["s2_periodic"])


def test_stream_3d(golden, mode):
    d = golden("percall")
    A = Args(mode)
    f, ct = A(d["s3_f"]), A(d["s3_ct"])
    out = A(np.zeros_like(d["s3_f"]))
    wb.lib.d3q19_stream_with_boundaries(A.ptr(f), A.ptr(out), A.ptr(ct), 10, 8, 6, 0.05, 0.0, 0.02)
    assert same_stream(A.np(out), d["s3_stream"])
    per = A(np.zeros_like(d["s3_f"]))
    wb.lib.d3q19_stream_periodic(A.ptr(f), A.ptr(per), 10, 8, 6)
    assert same_stream(A.np(per), d["s3_periodic"])
    f27 = A(d["s27_f"])
    p27 = A(np.zeros_like(d["s27_f"]))
    wb.lib.d3q27_stream_periodic(A.ptr(f27), A.ptr(p27), 10, 8, 6)
    assert same_stream(A.np(p27), d["s27_periodic"])


def test_zou_he_2d(golden, mode):
    d = golden("percall")
    A = Args(mode)
    n = 240
    f = A(d["s2_f"])
    rho, ux, uy = (A(np.zeros(n, np.float32)) for _ in range(3))
    wb.lib.d2q9_apply_zou_he_inflow_west(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), 0.05, 0.01, 20, 12)
    wb.lib.d2q9_apply_zou_he_outflow_east(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), 1.01, 20, 12)
    assert close(A.np(f), d["s2_zh_f"])
    assert close(A.np(rho), d["s2_zh_rho"])
    assert close(A.np(ux), d["s2_zh_ux"], 1e-5)
    assert close(A.np(uy), d["s2_zh_uy"], 1e-5)


def test_moments_speed_les_2d(golden, mode):
    d = golden("percall")
    A = Args(mode)
    n = 240
    f = A(d["s2_f"])
    rho, ux, uy, sp, te = (A(np.zeros(n, np.float32)) for _ in range(5))
    wb.lib.d2q9_compute_macroscopic_moments_forced(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), 1e-4, -2e-4, n)
    wb.lib.d2q9_compute_velocity_magnitude(A.ptr(ux), A.ptr(uy), A.ptr(sp), n)
    assert close(A.np(rho), d["s2_mf_rho"])
    assert close(A.np(ux), d["s2_mf_ux"], 1e-5) and close(A.np(uy), d["s2_mf_uy"], 1e-5)
    assert close(A.np(sp), d["s2_speed"], 1e-5)
    wb.lib.d2q9_compute_smagorinsky_tau(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), A.ptr(te), 0.52, 0.17, n)
    assert close(A.np(te), d["s2_tau_eff"])


def test_moments_les_3d(golden, mode):
    d = golden("percall")
    A = Args(mode)
    n = 480
    f = A(d["s3_f"])
    rho, ux, uy, uz, te = (A(np.zeros(n, np.float32)) for _ in range(5))
    wb.lib.d3q19_compute_macroscopic_moments(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), A.ptr(uz), n)
    for k, b in (("rho", rho), ("ux", ux), ("uy", uy), ("uz", uz)):
        assert close(A.np(b), d[f"s3_{k}"], 1e-5)
    wb.lib.d3q19_compute_smagorinsky_tau(A.ptr(f), A.ptr(rho), A.ptr(ux), A.ptr(uy), A.ptr(uz), A.ptr(te), 0.52, 0.17,
                                         n)
    assert close(A.np(te), d["s3_tau_eff"])


def test_momentum_exchange(golden, mode):
    d = golden("percall")
    A = Args(mode)
    out = [A(np.zeros(1, np.float32)) for _ in range(3)]
    f, ct = A(d["s2_f"]), A(d["s2_ct"])
    wb.lib.d2q9_compute_momentum_exchange_forces(A.ptr(f), A.ptr(ct), 20, 12, 8.5, 5.5, 4.0,
                                                 *[A.ptr(o) for o in out])
    got = np.array([A.np(o)[0] for o in out])
    assert np.allclose(got, d["s2_mem"], rtol=1e-5, atol=1e-6)
    out3 = [A(np.zeros(1, np.float32)) for _ in range(3)]
    f3, ct3 = A(d["s3_f"]), A(d["s3_ct"])
    wb.lib.d3q19_compute_momentum_exchange_forces(A.ptr(f3), A.ptr(ct3), 10, 8, 6, 4.5, 3.5, 2.5, 0.0,
                                                  *[A.ptr(o) for o in out3])
    got3 = np.array([A.np(o)[0] for o in out3])
    assert np.allclose(got3, d["s3_mem"], rtol=1e-5, atol=1e-6)


def test_momentum_exchange_kat(mode):
    """Known answers of tests/unit/test_forces_momentum_exchange.cpp:33-68."""
    A = Args(mode)
    nx = ny = 16
    w = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4, np.float32)
    f0 = np.repeat(w[:, None], nx * ny, axis=1)
    ct0 = np.zeros((ny, nx), np.uint8)
    ct0[7:9, 7:9] = 1
    f, ct = A(f0), A(ct0.ravel())
    out = [A(np.zeros(1, np.float32)) for _ in range(3)]
    wb.lib.d2q9_compute_momentum_exchange_forces(A.ptr(f), A.ptr(ct), nx, ny, 7.5, 7.5, 0.0, *[A.ptr(o) for o in out])
    assert abs(A.np(out[0])[0]) <= 1e-5 and abs(A.np(out[1])[0]) <= 1e-5
    f1 = f0.copy()
    f1[1, 7 * nx + 6] += 0.05
    f = A(f1)
    wb.lib.d2q9_compute_momentum_exchange_forces(A.ptr(f), A.ptr(ct), nx, ny, 7.5, 7.5, 0.0, *[A.ptr(o) for o in out])
    assert abs(A.np(out[0])[0] - 0.1) <= 1e-5


def test_curved_bfl(golden, mode):
    d = golden("percall")
    A = Args(mode)
    nl = len(d["s3_bfl_idx"])
    dst = A(d["s3_stream"])
    src = A(d["s3_f"])
    arrs = [A(d[k]) for k in ("s3_bfl_idx", "s3_bfl_q", "s3_bfl_delta", "s3_bfl_uwx")]
    zy, zz = A(np.zeros(nl, np.float32)), A(np.zeros(nl, np.float32))
    wb.lib.d3q19_apply_curved_bfl(A.ptr(dst), A.ptr(src), *[A.ptr(a) for a in arrs], A.ptr(zy), A.ptr(zz), 10, 8, 6,
                                  nl)
    assert close(A.np(dst), d["s3_bfl_out"])


def test_thermal(golden, mode):
    d = golden("percall")
    A = Args(mode)
    n = 96
    g, ct, ux, uy = A(d["th_g"]), A(d["th_ct"]), A(d["th_ux"]), A(d["th_uy"])
    out = A(np.zeros_like(d["th_g"]))
    T = A(np.zeros(n, np.float32))
    wb.lib.thermal_collide_d2q9(A.ptr(g), A.ptr(out), A.ptr(ct), A.ptr(ux), A.ptr(uy), A.ptr(T), 0.7, n)
    assert close(A.np(out), d["th_out"]) and close(A.np(T), d["th_T"])
    wb.lib.thermal_apply_isothermal_wall(A.ptr(out), 12, 8, 0, 1.0)
    assert close(A.np(out), d["th_wall"])
    gy = A(np.full(n, 1e-5, np.float32))
    wb.lib.thermal_compute_buoyancy_force_2d(A.ptr(T), A.ptr(gy), 0.5, 0.01, 0.1, n)
    assert close(A.np(gy), d["th_gy"])


def test_null_pointer_is_reported_not_faulted():
    wb.lib.wake_gpu_clear_error()
    wb.lib.d2q9_compute_macroscopic_moments(None, None, None, None, 16)
    assert wb.lib.wake_gpu_last_error_code() == -1
    wb.lib.wake_gpu_clear_error()


# ----------------------------------------------------------------------------- ragged and empty inputs
def _ref_lib():
    import oracle

    R = oracle.ref()
    if R is None:
        pytest.skip("reference build oracle/_ref is absent")
    vp, F, I = C.c_void_p, C.c_float, C.c_int
    R.d2q9_compute_macroscopic_moments.argtypes = [vp, vp, vp, vp, I]
    R.d2q9_collide_bgk.argtypes = [vp, vp, vp, vp, vp, vp, F, F, F, I]
    R.d3q19_collide_trt.argtypes = [vp, vp, vp, vp, vp, vp, vp, F, F, F, F, F, I]
    return R


def _pops(q, count, seed):
    import oracle

    rng = np.random.default_rng(seed)
    rho = (1.0 + 0.01 * rng.standard_normal(count)).astype(np.float32)
    u = [(0.03 * rng.standard_normal(count)).astype(np.float32) for _ in range(3)]
    f = oracle.equilibrium(q, rho, u[0], u[1], u[2] if q != 9 else None, prec=32)
    return np.ascontiguousarray((f * (1.0 + 0.01 * rng.standard_normal(f.shape))).astype(np.float32))


@pytest.mark.parametrize("count", [1, 33, 257, 4099])
def test_ragged_counts_match_reference(mode, count):
    """Node counts that fill no whole block: the last block's tail must be neither skipped nor
    overrun. Moments, BGK (D2Q9) and TRT (D3Q19) collide against the reference's kernels."""
    R = _ref_lib()
    A = Args(mode)
    types = np.zeros(count, np.uint8)
    types[::7] = 1  # some solids (copied through)
    f9 = _pops(9, count, count)
    want = [np.zeros(count, np.float32) for _ in range(3)]
    R.d2q9_compute_macroscopic_moments(f9.ctypes.data, *[w.ctypes.data for w in want], count)
    got = [A(np.full(count, np.nan, np.float32)) for _ in range(3)]
    wb.lib.d2q9_compute_macroscopic_moments(A.ptr(A(f9)), *[A.ptr(g) for g in got], count)
    for g, w in zip(got, want):
        assert close(A.np(g), w)
    fo_ref = np.zeros_like(f9)
    mom = [np.zeros(count, np.float32) for _ in range(3)]
    R.d2q9_collide_bgk(f9.ctypes.data, fo_ref.ctypes.data, types.ctypes.data, *[m.ctypes.data for m in mom], 0.7,
                       0.0, 0.0, count)
    fo = A(np.zeros_like(f9))
    gm = [A(np.zeros(count, np.float32)) for _ in range(3)]
    wb.lib.d2q9_collide_bgk(A.ptr(A(f9)), A.ptr(fo), A.ptr(A(types)), *[A.ptr(m) for m in gm], 0.7, 0.0, 0.0, count)
    assert close(A.np(fo), fo_ref)
    f19 = _pops(19, count, count + 1)
    fo_ref = np.zeros_like(f19)
    mom = [np.zeros(count, np.float32) for _ in range(4)]
    R.d3q19_collide_trt(f19.ctypes.data, fo_ref.ctypes.data, types.ctypes.data, *[m.ctypes.data for m in mom], 0.75,
                        1.3, 0.0, 0.0, 0.0, count)
    fo = A(np.zeros_like(f19))
    gm = [A(np.zeros(count, np.float32)) for _ in range(4)]
    wb.lib.d3q19_collide_trt(A.ptr(A(f19)), A.ptr(fo), A.ptr(A(types)), *[A.ptr(m) for m in gm], 0.75, 1.3, 0.0,
                             0.0, 0.0, count)
    assert close(A.np(fo), fo_ref)


def test_empty_inputs_touch_nothing(mode):
    """Zero-sized calls (count 0, an extent of 0) return without writing, as the reference's
    loops over empty ranges do, and record no error."""
    A = Args(mode)
    wb.lib.wake_gpu_clear_error()
    sentinel = np.full(64, 7.0, np.float32)
    bufs = [A(sentinel) for _ in range(6)]
    t = A(np.zeros(64, np.uint8))
    p = [A.ptr(b) for b in bufs]
    wb.lib.d2q9_compute_macroscopic_moments(p[0], p[1], p[2], p[3], 0)
    wb.lib.d2q9_collide_bgk(p[0], p[1], A.ptr(t), p[2], p[3], p[4], 0.7, 0.0, 0.0, 0)
    wb.lib.d2q9_stream_periodic(p[0], p[1], 0, 4)
    wb.lib.d3q19_stream_periodic(p[0], p[1], 4, 0, 2)
    wb.lib.d3q19_apply_curved_bfl(p[0], p[1], None, None, None, None, None, None, 4, 4, 4, 0)
    wb.lib.compute_vorticity_2d(p[0], p[1], p[2], 0, 8)
    wb.lib.compute_vorticity_and_q_criterion_3d(p[0], p[1], p[2], p[3], p[4], p[5], p[5], 4, 4, 0)
    for b in bufs:
        assert np.array_equal(A.np(b), sentinel)
    assert wb.lib.wake_gpu_last_error_code() == 0


def test_immersed_boundary_against_reference(mode):
    """Velocity interpolation to markers and force spreading (Roma-Peskin delta) against the
    reference's own kernels (src/ispc/ibm_kernels.ispc), with markers near the x wrap and the
    y edges. Spreading adds overlapping markers with atomics, so it matches to rounding."""
    R = _ref_lib()
    vp, I = C.c_void_p, C.c_int
    R.ibm_interpolate_velocity_2d.argtypes = [vp, vp, vp, vp, vp, vp, I, I, I]
    R.ibm_spread_force_2d.argtypes = [vp, vp, vp, vp, vp, vp, vp, I, I, I]
    rng = np.random.default_rng(5)
    nx, ny, nm = 48, 32, 97
    ux = (0.05 * rng.standard_normal(nx * ny)).astype(np.float32)
    uy = (0.05 * rng.standard_normal(nx * ny)).astype(np.float32)
    theta = np.linspace(0.0, 2.0 * np.pi, nm, endpoint=False)
    mx = (24.0 + 9.5 * np.cos(theta)).astype(np.float32)
    my = (16.0 + 9.5 * np.sin(theta)).astype(np.float32)
    mx[:4] = [0.3, 47.6, 1.9, 46.2]  # across the periodic x wrap
    my[:4] = [0.4, 31.2, 1.1, 30.8]  # rows of the stencil outside [0, ny)
    fx = (1e-3 * rng.standard_normal(nm)).astype(np.float32)
    fy = (1e-3 * rng.standard_normal(nm)).astype(np.float32)
    ds = np.full(nm, 0.6, np.float32)
    want_u, want_v = np.zeros(nm, np.float32), np.zeros(nm, np.float32)
    R.ibm_interpolate_velocity_2d(ux.ctypes.data, uy.ctypes.data, mx.ctypes.data, my.ctypes.data,
                                  want_u.ctypes.data, want_v.ctypes.data, nx, ny, nm)
    A = Args(mode)
    gu, gv = A(np.full(nm, np.nan, np.float32)), A(np.full(nm, np.nan, np.float32))
    wb.lib.ibm_interpolate_velocity_2d(A.ptr(A(ux)), A.ptr(A(uy)), A.ptr(A(mx)), A.ptr(A(my)), A.ptr(gu), A.ptr(gv),
                                       nx, ny, nm)
    assert close(A.np(gu), want_u) and close(A.np(gv), want_v)
    gx0 = (1e-6 * rng.standard_normal(nx * ny)).astype(np.float32)
    gy0 = (1e-6 * rng.standard_normal(nx * ny)).astype(np.float32)
    want_gx, want_gy = gx0.copy(), gy0.copy()
    R.ibm_spread_force_2d(mx.ctypes.data, my.ctypes.data, fx.ctypes.data, fy.ctypes.data, ds.ctypes.data,
                          want_gx.ctypes.data, want_gy.ctypes.data, nx, ny, nm)
    ggx, ggy = A(gx0), A(gy0)
    wb.lib.ibm_spread_force_2d(A.ptr(A(mx)), A.ptr(A(my)), A.ptr(A(fx)), A.ptr(A(fy)), A.ptr(A(ds)), A.ptr(ggx),
                               A.ptr(ggy), nx, ny, nm)
    assert close(A.np(ggx), want_gx) and close(A.np(ggy), want_gy)
