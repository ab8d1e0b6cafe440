"""Field analytics (vorticity, Q-criterion) and VTK files.

CPU: the oracle's restatement of src/ispc/analytics_kernels.ispc against the
reference's own kernels (translated and compiled into oracle/_ref), and the
library's VTK writers against the reference's VtkExporter on the same fields,
byte for byte. GPU: the device kernels (drop-in and engine) against the oracle,
bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

import oracle

REF = oracle.ref()
needs_ref = pytest.mark.skipif(REF is None, reason="reference build oracle/_ref is absent")


def _fields(n, seed, k=3, scale=0.05):
    rng = np.random.default_rng(seed)
    return [(scale * rng.standard_normal(n)).astype(np.float32) for _ in range(k)]


def _q_scale(ux, uy, uz, nx, ny, nz):
    """Per node |Omega|^2 + |S|^2 (FP64), the size Q is a difference of."""
    u = [a.astype(np.float64).reshape(nz, ny, nx) for a in (ux, uy, uz)]
    g = [[0.5 * (np.roll(a, -1, ax) - np.roll(a, 1, ax)) for ax in (2, 1, 0)] for a in u]
    return sum(g[i][j] ** 2 for i in range(3) for j in range(3)).ravel()


# ----------------------------------------------------------------------------- CPU: oracle pins
@needs_ref
@pytest.mark.parametrize("nx,ny", [(37, 23), (1, 5), (64, 1), (3, 3)])
def test_oracle_vorticity_2d_equals_reference_kernel(nx, ny):
    ux, uy = _fields(nx * ny, nx + 7 * ny, 2)
    ref = np.empty(nx * ny, np.float32)
    REF.compute_vorticity_2d(ux.ctypes.data, uy.ctypes.data, ref.ctypes.data, nx, ny)
    assert np.array_equal(ref, oracle.vorticity_2d(ux, uy, nx, ny))


@needs_ref
@pytest.mark.parametrize("nx,ny,nz", [(19, 13, 11), (4, 1, 6), (2, 2, 2)])
def test_oracle_vorticity_q_3d_matches_reference_kernel(nx, ny, nz):
    """Vorticity is bit-identical. Q is a difference of two sums of squares, and the reference's
    fast-math build contracts and reorders them: the two agree to a few ulp of |Omega|^2 + |S|^2."""
    n = nx * ny * nz
    u = _fields(n, n, 3)
    out = [np.empty(n, np.float32) for _ in range(4)]
    REF.compute_vorticity_and_q_criterion_3d(*[a.ctypes.data for a in u], *[a.ctypes.data for a in out], nx, ny, nz)
    mine = oracle.vorticity_q_3d(*u, nx, ny, nz)
    for a, b in zip(out[:3], mine[:3]):
        assert np.array_equal(a, b)
    bound = 2.0 ** -20 * _q_scale(*u, nx, ny, nz) + 1e-30
    assert np.all(np.abs(out[3].astype(np.float64) - mine[3]) <= bound)
    # and the FP32 restatement is within FP32 rounding of the FP64 one
    q64 = oracle.vorticity_q_3d(*u, nx, ny, nz, dtype=np.float64)[3]
    assert np.all(np.abs(mine[3] - q64) <= bound)


# ----------------------------------------------------------------------------- CPU: VTK bytes
def _ref_grid_2d(nx=40, ny=24, steps=30):
    g = oracle.RefGrid2D(nx, ny, 0.56)
    n = nx * ny
    ux, uy = _fields(n, 5, 2, 0.01)
    g.init_fields(np.ones(n, np.float32), ux + np.float32(0.05), uy)
    REF.ref2d_set_solid_circle(g._h, 12.0, 12.0, 4.0)
    REF.ref2d_set_inflow_west(g._h, 0.05, 0.0)
    REF.ref2d_set_outflow_east(g._h, 1.0)
    g.step(steps, 0)
    return g


@needs_ref
@pytest.mark.parametrize("with_vorticity", [True, False])
def test_vti_2d_bytes_equal_reference(tmp_path, with_vorticity):
    import wake_b200 as wb

    g = _ref_grid_2d()
    nx, ny = g.nx, g.ny
    m = g.macro()
    t = g.cell_types()
    vort = oracle.vorticity_2d(m["ux"], m["uy"], nx, ny) if with_vorticity else None
    ref_path, ours = tmp_path / "ref.vti", tmp_path / "ours.vti"
    assert REF.ref_vtk_export_2d(g._h, str(ref_path).encode(), vort.ctypes.data if vort is not None else None) == 0
    for threads in (1, 7):
        assert wb.lib.wake_vtk_write_vti_2d(str(ours).encode(), nx, ny, m["ux"].ctypes.data, m["uy"].ctypes.data,
                                            m["speed"].ctypes.data, m["rho"].ctypes.data,
                                            vort.ctypes.data if vort is not None else None, t.ctypes.data,
                                            threads) == 0
        assert ours.read_bytes() == ref_path.read_bytes()


@needs_ref
def test_vti_3d_bytes_equal_reference(tmp_path):
    import wake_b200 as wb

    nx, ny, nz = 14, 10, 8
    n = nx * ny * nz
    g = oracle.RefGrid3D(nx, ny, nz, 0.6)
    ux, uy, uz = _fields(n, 11, 3, 0.01)
    g.init_fields(np.ones(n, np.float32), ux + np.float32(0.03), uy, uz)
    REF.ref3d_set_periodic(g._h, 1)
    REF.ref3d_set_solid_sphere(g._h, 6.0, 5.0, 4.0, 2.5)
    g.step(10, 1)
    m = g.macro()
    t = g.cell_types()
    wx, wy, wz, q = oracle.vorticity_q_3d(m["ux"], m["uy"], m["uz"], nx, ny, nz)
    inter = np.ascontiguousarray(np.stack([wx, wy, wz], axis=1))
    cases = [("all", q, (wx, wy, wz), inter), ("q", q, (None,) * 3, None), ("none", None, (None,) * 3, None)]
    for name, qq, w, wi in cases:
        ref_path, ours = tmp_path / f"ref_{name}.vti", tmp_path / f"ours_{name}.vti"
        assert REF.ref_vtk_export_3d(g._h, str(ref_path).encode(), qq.ctypes.data if qq is not None else None,
                                     wi.ctypes.data if wi is not None else None) == 0
        assert wb.lib.wake_vtk_write_vti_3d(str(ours).encode(), nx, ny, nz, m["ux"].ctypes.data,
                                            m["uy"].ctypes.data, m["uz"].ctypes.data, m["speed"].ctypes.data,
                                            m["rho"].ctypes.data, qq.ctypes.data if qq is not None else None,
                                            *[c.ctypes.data if c is not None else None for c in w], t.ctypes.data,
                                            3) == 0
        assert ours.read_bytes() == ref_path.read_bytes(), name


@needs_ref
@pytest.mark.parametrize("start,end,every,dt", [(0, 1000, 100, 1.0), (-20, 35, 7, 0.37), (5, 4, 1, 2.0),
                                                (999990, 1000010, 10, 1e-3)])
def test_pvd_bytes_equal_reference(tmp_path, start, end, every, dt):
    import wake_b200 as wb

    ref_path, ours = tmp_path / "ref.pvd", tmp_path / "ours.pvd"
    assert REF.ref_vtk_pvd(str(ref_path).encode(), b"frames/wake", start, end, every, dt) == 0
    assert wb.lib.wake_vtk_write_pvd(str(ours).encode(), b"frames/wake", start, end, every, dt) == 0
    assert ours.read_bytes() == ref_path.read_bytes()


def test_vtk_writer_rejects_bad_arguments(tmp_path):
    import wake_b200 as wb

    x = np.zeros(4, np.float32)
    t = np.zeros(4, np.uint8)
    assert wb.lib.wake_vtk_write_vti_2d(str(tmp_path / "a.vti").encode(), 0, 4, *[x.ctypes.data] * 4, None,
                                        t.ctypes.data, 1) < 0
    assert wb.lib.wake_vtk_write_vti_2d(str(tmp_path / "no_dir" / "a.vti").encode(), 2, 2, *[x.ctypes.data] * 4,
                                        None, t.ctypes.data, 1) < 0
    assert wb.lib.wake_vtk_write_vti_3d(str(tmp_path / "b.vti").encode(), 1, 2, 2, *[x.ctypes.data] * 5, None,
                                        x.ctypes.data, None, None, t.ctypes.data, 1) < 0
    assert wb.lib.wake_vtk_write_pvd(str(tmp_path / "c.pvd").encode(), b"p", 0, 10, 0, 1.0) < 0
    wb.lib.wake_gpu_clear_error()


# ----------------------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(37, 23), (1, 5), (300, 70000)])
def test_dropin_vorticity_2d_bit_exact(nx, ny):
    import torch

    import wake_b200 as wb

    ux, uy = _fields(nx * ny, 3, 2)
    want = oracle.vorticity_2d(ux, uy, nx, ny)
    v = np.full(nx * ny, np.nan, np.float32)
    wb.lib.compute_vorticity_2d(ux.ctypes.data, uy.ctypes.data, v.ctypes.data, nx, ny)  # host buffers, staged
    assert np.array_equal(v, want)
    d = [torch.from_numpy(a).cuda() for a in (ux, uy)]
    out = torch.full((nx * ny,), float("nan"), device="cuda")
    wb.lib.compute_vorticity_2d(d[0].data_ptr(), d[1].data_ptr(), out.data_ptr(), nx, ny)  # device, in place
    assert np.array_equal(out.cpu().numpy(), want)
    assert wb.FieldAnalytics.compute_max_vorticity_2d(out) == np.float32(np.abs(want).max())
    assert wb.FieldAnalytics.compute_max_vorticity_2d(v) == np.float32(np.abs(want).max())


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,nz", [(19, 13, 11), (4, 1, 6), (130, 66, 40)])
def test_dropin_vorticity_q_3d_bit_exact(nx, ny, nz):
    import torch

    import wake_b200 as wb

    n = nx * ny * nz
    u = _fields(n, 17, 3)
    want = oracle.vorticity_q_3d(*u, nx, ny, nz)
    out = [np.full(n, np.nan, np.float32) for _ in range(4)]
    wb.lib.compute_vorticity_and_q_criterion_3d(*[a.ctypes.data for a in u], *[a.ctypes.data for a in out], nx, ny, nz)
    for a, b in zip(out, want):
        assert np.array_equal(a, b)
    du = [torch.from_numpy(a).cuda() for a in u]
    dout = [torch.full((n,), float("nan"), device="cuda") for _ in range(4)]
    wb.lib.compute_vorticity_and_q_criterion_3d(*[a.data_ptr() for a in du], *[a.data_ptr() for a in dout], nx, ny,
                                                nz)
    for a, b in zip(dout, want):
        assert np.array_equal(a.cpu().numpy(), b)


@pytest.mark.gpu
def test_abs_max_skips_nan_and_handles_empty():
    import torch

    import wake_b200 as wb

    v = torch.tensor([0.5, float("nan"), -3.25, 1.0, float("-inf")], device="cuda")
    assert wb.FieldAnalytics.compute_max_vorticity_2d(v) == float("inf")
    v = torch.tensor([0.5, float("nan"), -3.25, 1.0], device="cuda")
    assert wb.FieldAnalytics.compute_max_vorticity_2d(v) == 3.25
    assert wb.FieldAnalytics.compute_max_vorticity_2d(torch.empty(0, device="cuda")) == 0.0
    assert wb.FieldAnalytics.compute_max_vorticity_2d(np.array([-0.0], np.float32)) == 0.0


@pytest.mark.gpu
def test_grid_analytics_equal_oracle_on_the_grids_moments(tmp_path):
    """The engine's analytics read the resident moments: equal, bit for bit, to the oracle's
    stencil applied to the moments the grid reports; the export writes those same values."""
    import wake_b200 as wb
    from wake_b200 import workloads as W

    c = W.cylinder_channel(nx=200, ny=80, diameter=10.0, cx=40.0, cy=40.0)
    g = W.build_grid(c)
    g.step(c.collision, n=300)
    m = g.macroscopic()
    want = oracle.vorticity_2d(m["ux"], m["uy"], g.nx, g.ny)
    got = wb.FieldAnalytics.compute_vorticity(g)
    assert np.array_equal(got, want)
    dev = wb.FieldAnalytics.compute_vorticity(g, device=True)
    assert np.array_equal(dev.cpu().numpy(), want)
    assert wb.FieldAnalytics.max_vorticity(g) == np.float32(np.abs(want).max())
    a, b = tmp_path / "grid.vti", tmp_path / "host.vti"
    wb.VtkExporter.export_grid(str(a), g)
    assert wb.VtkExporter.export_vti_2d(str(b), g, vorticity=want)
    assert a.read_bytes() == b.read_bytes()
    g.close()

    s = W.sphere_channel(nx=64, ny=32, nz=32, radius=5.0, center=(16.0, 16.0, 16.0))
    g = W.build_grid(s)
    g.step(s.collision, use_les=s.les, smag_const=s.cs_smag, n=100)
    m = g.macroscopic()
    want = oracle.vorticity_q_3d(m["ux"], m["uy"], m["uz"], g.nx, g.ny, g.nz)
    got = wb.FieldAnalytics.compute_3d_features(g)
    for x, y in zip(got, want):
        assert np.array_equal(x, y)
    a, b = tmp_path / "grid3.vti", tmp_path / "host3.vti"
    wb.VtkExporter.export_grid(str(a), g)
    assert wb.VtkExporter.export_vti_3d(str(b), g, q_criterion=want[3], vorticity=want[:3])
    assert a.read_bytes() == b.read_bytes()
    g.close()


@pytest.mark.gpu
@needs_ref
def test_dropin_vorticity_on_reference_fields_equals_reference():
    """FieldAnalytics::compute_vorticity's kernel on a reference grid's own velocity: the GPU drop-in
    gives the reference's bytes."""
    import wake_b200 as wb

    g = _ref_grid_2d(64, 40, 60)
    m = g.macro()
    ref = np.empty(g.nx * g.ny, np.float32)
    REF.compute_vorticity_2d(m["ux"].ctypes.data, m["uy"].ctypes.data, ref.ctypes.data, g.nx, g.ny)
    ours = np.empty_like(ref)
    wb.lib.compute_vorticity_2d(m["ux"].ctypes.data, m["uy"].ctypes.data, ours.ctypes.data, g.nx, g.ny)
    assert np.array_equal(ours, ref)
