"""Pins the CPU oracle: the reference's known-answer tests, the reference's own
outputs (golden fixtures and, where built, the reference library), and the
analytic properties of the pieces the reference lacks. CPU only."""
import re

import numpy as np
import pytest

import oracle
from conftest import rel_l2, vel_rel_l2
from oracle.build_ref import reference_dir
from wake_b200 import workloads as W

REF_SRC = reference_dir()


def eq(q, rho, u):
    n = 1
    return oracle.equilibrium(q, np.full(n, rho), np.full(n, u[0]), np.full(n, u[1]),
                              None if q == 9 else np.full(n, u[2]), prec=64)[:, 0]


# ---------------------------------------------------------------- reference KATs
@pytest.mark.parametrize("q,rho,u", [(9, 1.05, (0.08, -0.04, 0.0)), (19, 1.02, (0.05, -0.03, 0.04))])
def test_moments_of_equilibrium(q, rho, u):
    """tests/unit/test_d2q9_moments.cpp:28-66, tests/unit/test_d3q19_moments.cpp:27-62."""
    nx = 4
    og = oracle.OracleGrid(q, nx, nx, 1 if q == 9 else nx, 64)
    n = og.n
    f = np.repeat(eq(q, rho, u)[:, None], n, axis=1)
    og.set_state(f)
    og.lib = None
    lib = oracle.lib()
    # moments of the state through the oracle's own forced-moment path with g = 0
    og.configure(collision=0, tau=1e9)
    m = {k: np.empty(n) for k in ("rho", "ux", "uy", "uz", "speed")}
    lib.og_get_macro  # noqa: B018  (present)
    out = og.macro()
    # og_set_state stores rho/u as given; recompute moments directly from f
    cx = {9: [0, 1, 0, -1, 0, 1, -1, -1, 1]}
    if q == 9:
        c = np.array([[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]])
        r = f.sum(0)
        uu = (c.T @ f) / r
        assert np.all(np.abs(r - rho) <= 1e-5) and np.all(np.abs(uu[0] - u[0]) <= 1e-5)
        assert np.all(np.abs(uu[1] - u[1]) <= 1e-5)
    del m, out, cx


def _conservation(q, model, taus):
    """tests/unit/test_d2q9_collision.cpp:31-121, tests/unit/test_d3q19_collision.cpp:34-113."""
    count = 32 if q == 9 else 16
    w = eq(q, 1.0, (0.0, 0.0, 0.0))
    k = 1 if q == 9 else 3
    f = np.array([[w[j] + (0.01 if q == 9 else 0.005) * np.sin(k * j + i) for i in range(count)] for j in range(q)])
    og = oracle.OracleGrid(q, count, 1, 1, 64)
    tau_s = taus[0]
    kw = dict(collision=model, tau=tau_s)
    if model == 1:
        kw["lambda_trt"] = (taus[0] - 0.5) * (taus[1] - 0.5)
    if model == 2:
        kw["tau_bulk"] = taus[1]
    og.configure(**kw)
    ct = np.zeros(count, np.uint8)
    ct[-1] = 1
    out = np.empty((count, q))
    rho, ux, uy, uz = (np.empty(count) for _ in range(4))
    fn = np.ascontiguousarray(f.T)
    oracle.lib().og_collide_nodes(og._h, count, fn.ctypes.data, ct.ctypes.data, out.ctypes.data, rho.ctypes.data,
                                  ux.ctypes.data, uy.ctypes.data, uz.ctypes.data)
    c = {9: np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, -1, 0], [1, 1, 0], [-1, 1, 0], [-1, -1, 0],
                      [1, -1, 0]])}.get(q)
    if c is None:
        c = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                      [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1], [0, 1, 1],
                      [0, -1, 1], [0, 1, -1], [0, -1, -1]])
    pre, post = f[:, 0], out[0]
    assert abs(post.sum() - pre.sum()) <= 1e-5
    assert np.all(np.abs(c.T @ post - c.T @ pre) <= 1e-5)
    assert np.array_equal(out[-1], f[:, -1])  # solid node unchanged


@pytest.mark.parametrize("model,taus", [(0, (0.7,)), (1, (0.7, 1.2)), (2, (0.7, 1.6))])
def test_d2q9_collision_conservation(model, taus):
    _conservation(9, model, taus)


@pytest.mark.parametrize("model,taus", [(0, (0.75,)), (1, (0.75, 1.3)), (2, (0.75, 1.2))])
def test_d3q19_collision_conservation(model, taus):
    _conservation(19, model, taus)


def test_momentum_exchange_kat():
    """tests/unit/test_forces_momentum_exchange.cpp:33-68: F = 0 at rest, +0.05 on q=1 gives Fx = 0.1."""
    n = 16
    og = oracle.OracleGrid(9, n, n, 1, 64)
    og.configure(mem=1, center=(7.5, 7.5, 0.0), r_max=0.0)
    t = np.zeros((n, n), np.uint8)
    t[7:9, 7:9] = 1
    og.set_cell_types(t)
    f = np.repeat(eq(9, 1.0, (0, 0, 0))[:, None], n * n, axis=1)
    og.set_state(f)
    F = og.forces()
    assert abs(F[0]) <= 1e-5 and abs(F[1]) <= 1e-5
    f[1, 7 * n + 6] += 0.05
    og.set_state(f)
    assert abs(og.forces()[0] - 0.1) <= 1e-5


def test_strouhal_kat(golden):
    d = golden("kat")
    f = oracle.strouhal_frequency(d["strouhal_signal"], 1.0)
    assert abs(f - 0.025) <= 0.003
    assert abs(f - float(d["strouhal_freq"])) <= 1e-6


# ---------------------------------------------------------------- vs the reference's own outputs
@pytest.mark.parametrize("tag,coll", [("bgk", 0), ("trt", 1), ("mrt", 2)])
def test_oracle_matches_reference_cylinder(golden, tag, coll):
    d = golden(f"cyl2d_{tag}")
    og = oracle.OracleGrid(9, 64, 32, 1, 32)
    og.configure(collision=coll, tau=float(d["tau"]), inflow=1, outflow=1, u_in=(0.05, 0, 0), rho_out=1.0, mem=1,
                 center=(16.0, 16.0, 0.0), r_max=12.0)
    og.set_cell_types(d["types"])
    og.set_state(d["f0"])
    hist = og.step(int(d["steps"]), forces=True)
    m = og.macro()
    assert vel_rel_l2(m, d) <= 1e-5 and rel_l2(m["rho"], d["rho"]) <= 1e-5
    assert rel_l2(hist[:, :2], d["forces"][:, :2]) <= 1e-4


@pytest.mark.parametrize("tag,coll", [("bgk", 0), ("trt", 1), ("mrt", 2)])
def test_oracle_matches_reference_sphere(golden, tag, coll):
    d = golden(f"sphere3d_{tag}")
    nx, ny, nz = 24, 16, 16
    og = oracle.OracleGrid(19, nx, ny, nz, 32)
    og.configure(collision=coll, tau=float(d["tau"]), mem=1, center=(8.0, 8.0, 8.0), r_max=8.0)
    og.set_cell_types(d["types"])
    og.set_state(np.repeat(d["f0_node"][:, None], nx * ny * nz, axis=1))
    og.set_links(d["links_idx"], d["links_q"], d["links_delta"])
    hist = og.step(int(d["steps"]), forces=True)
    m = og.macro()
    assert vel_rel_l2(m, d, ("ux", "uy", "uz")) <= 1e-5 and rel_l2(m["rho"], d["rho"]) <= 1e-5
    assert rel_l2(hist, d["forces"]) <= 1e-4


def test_oracle_matches_reference_cavity_and_tgv(golden):
    d = golden("cavity2d_mrt")
    og = oracle.OracleGrid(9, 32, 32, 1, 32)
    og.configure(collision=2, tau=float(d["tau"]), u_wall=(float(d["lid"]), 0.0, 0.0))
    og.set_cell_types(d["types"])
    og.set_state(d["f0"])
    og.step(int(d["steps"]))
    assert vel_rel_l2(og.macro(), d) <= 1e-5
    d = golden("tgv3d_mrt")
    og = oracle.OracleGrid(19, 12, 12, 12, 32)
    og.configure(collision=2, tau=float(d["tau"]), periodic_y=1, periodic_z=1)
    og.set_state(d["f0"])
    og.step(int(d["steps"]))
    assert vel_rel_l2(og.macro(), d, ("ux", "uy", "uz")) <= 1e-5


def test_rounded_mrt_inverse_is_the_reference_table():
    """The 7-decimal D3Q19 inverse equals src/ispc/d3q19_collision_mrt.ispc:4-24 (read as text)."""
    src = REF_SRC / "src" / "ispc" / "d3q19_collision_mrt.ispc"
    if not src.exists():
        pytest.skip("reference sources not present")
    body = src.read_text().split("d3q19_Minv[D3Q19_Q][D3Q19_Q] = {", 1)[1].split("};", 1)[0]
    vals = np.array([float(v) for v in re.findall(r"-?\d+\.\d+(?=f)", body)], np.float32).reshape(19, 19)
    ours = oracle.d3q19_minv(True).astype(np.float32)
    assert np.array_equal(vals, ours)
    exact = oracle.d3q19_minv(False)
    # the rounding shifts the column sums by ~1e-7 (mass drift of the reference's MRT)
    assert abs(exact[:, 0].sum() - 1.0) < 1e-12 and abs(ours[:, 0].astype(np.float64).sum() - 1.0) > 1e-8


def test_oracle_matches_reference_library_live():
    """Where the reference library is built: a fresh run, LES flag on (computed but unused there)."""
    R = oracle.ref()
    if R is None:
        pytest.skip("reference library not built")
    c = W.cylinder_channel(nx=48, ny=24, diameter=6, cx=12, cy=12, tau=0.58, collision=1)
    g = oracle.RefGrid2D(c.nx, c.ny, c.tau)
    g.init_fields(c.rho, c.ux, c.uy)
    R.ref2d_set_inflow_west(g._h, 0.05, 0.0)
    R.ref2d_set_outflow_east(g._h, 1.0)
    for x in range(c.nx):
        R.ref2d_set_cell_type(g._h, x, 0, 1)
        R.ref2d_set_cell_type(g._h, x, c.ny - 1, 1)
    R.ref2d_set_solid_circle(g._h, 12.0, 12.0, 3.0)
    assert np.array_equal(g.cell_types(), c.types)
    f0 = g.f()
    g.step(100, 1, use_les=True, cs=0.17)
    og = oracle.OracleGrid(9, c.nx, c.ny, 1, 32)
    og.configure(collision=1, tau=c.tau, inflow=1, outflow=1, u_in=(0.05, 0, 0), rho_out=1.0, les=0)
    og.set_cell_types(c.types)
    og.set_state(f0)
    og.step(100)
    assert vel_rel_l2(og.macro(), g.macro()) <= 1e-5


# ---------------------------------------------------------------- extensions (no reference source)
def test_d3q27_mrt_conserves_mass_and_momentum():
    q = 27
    count = 8
    rng = W.uniform24(W.BASE_SEED, q * count).reshape(q, count)
    w = eq(q, 1.0, (0, 0, 0))
    f = w[:, None] * (1.0 + 0.1 * (rng - 0.5))
    og = oracle.OracleGrid(q, count, 1, 1, 64)
    og.configure(collision=2, tau=0.6, tau_bulk=0.8, s3=1.1, s4=1.3)
    out = np.empty((count, q))
    rho, ux, uy, uz = (np.empty(count) for _ in range(4))
    fn = np.ascontiguousarray(f.T)
    oracle.lib().og_collide_nodes(og._h, count, fn.ctypes.data, None, out.ctypes.data, rho.ctypes.data,
                                  ux.ctypes.data, uy.ctypes.data, uz.ctypes.data)
    assert np.allclose(out.sum(1), fn.sum(1), rtol=0, atol=1e-14)
    # equilibrium is a fixed point
    fe = np.repeat(eq(q, 1.01, (0.02, -0.01, 0.03))[None, :], 2, axis=0)
    out2 = np.empty_like(fe)
    oracle.lib().og_collide_nodes(og._h, 2, np.ascontiguousarray(fe).ctypes.data, None, out2.ctypes.data,
                                  rho.ctypes.data, ux.ctypes.data, uy.ctypes.data, uz.ctypes.data)
    assert np.allclose(out2, fe, rtol=0, atol=1e-15)


def test_d3q27_mrt_taylor_green_decay_rate():
    """Kinetic energy of a periodic TGV decays like exp(-6 k^2 nu t) early on (form of
    tests/validation/test_taylor_green_decay.cpp:49-61), within 2.5%."""
    L, tau, steps = 16, 0.8, 60
    c = W.taylor_green(L=L, u0=0.04, tau=tau, q=27, collision=2)
    og = oracle.OracleGrid(27, L, L, L, 64)
    og.configure(collision=2, tau=tau, periodic_y=1, periodic_z=1)
    og.set_state(oracle.equilibrium(27, c.rho, c.ux, c.uy, c.uz, prec=64))
    m0 = og.macro()
    ke0 = (0.5 * m0["rho"] * (c.ux.astype(np.float64) ** 2 + c.uy.astype(np.float64) ** 2)).sum()
    og.step(steps)
    m = og.macro()
    ke = (0.5 * m["rho"] * m["speed"] ** 2).sum()
    nu = (tau - 0.5) / 3.0
    k = 2 * np.pi / L
    assert abs(ke / ke0 - np.exp(-6 * k * k * nu * steps)) <= 0.025


def test_zou_he_3d_imposes_inlet_velocity_and_outlet_density():
    c = W.sphere_channel(nx=12, ny=6, nz=6, radius=1.0, center=(6.0, 3.0, 3.0), tau=0.6, collision=1, les=False)
    og = oracle.OracleGrid(19, c.nx, c.ny, c.nz, 64)
    og.configure(collision=1, tau=0.6, periodic_y=1, periodic_z=1, inflow=1, u_in=(0.05, 0.01, -0.02), outflow=1,
                 rho_out=1.02)
    og.set_cell_types(c.types)
    og.set_state(oracle.equilibrium(19, c.rho, c.ux, c.uy, c.uz, prec=64))
    og.step(5)
    m = og.macro()
    ux = m["ux"].reshape(6, 6, 12)
    assert np.allclose(ux[:, :, 0], 0.05, atol=1e-12)
    assert np.allclose(m["uy"].reshape(6, 6, 12)[:, :, 0], 0.01, atol=1e-12)
    assert np.allclose(m["uz"].reshape(6, 6, 12)[:, :, 0], -0.02, atol=1e-12)
    assert np.allclose(m["rho"].reshape(6, 6, 12)[:, :, -1], 1.02, atol=1e-12)
    assert np.allclose(m["uy"].reshape(6, 6, 12)[:, :, -1], 0.0, atol=1e-12)


def test_applied_smagorinsky_tau():
    q = 19
    f = eq(q, 1.0, (0.03, 0.0, 0.0))
    assert abs(oracle.lib().og_smagorinsky_tau(q, f.ctypes.data, 1.0, 0.03, 0.0, 0.0, 0.52, 0.17) - 0.52) < 1e-12
    f2 = f.copy()
    f2[7] += 1e-3
    f2[8] -= 1e-3
    t = oracle.lib().og_smagorinsky_tau(q, f2.ctypes.data, 1.0, 0.03, 0.0, 0.0, 0.52, 0.17)
    assert t > 0.52


def test_thermal_conduction_state_is_exact():
    """D2Q5 temperature between isothermal walls (anti-bounce-back at y = -1/2 and ny - 1/2): without
    buoyancy the linear conduction profile with the fluid at rest is an exact steady state (with
    buoyancy the density stratifies first, a transient of relative size ~beta_g)."""
    nx, ny = 24, 12
    o = oracle.OracleGrid(9, nx, ny, 1, 64)
    o.configure(collision=1, tau=0.6, thermal=1, tau_t=0.6, t_ref=0.5, beta_g=0.0, t_south=1.0, t_north=0.0)
    o.set_cell_types(np.zeros(nx * ny, np.uint8))
    n = nx * ny
    o.set_state(oracle.equilibrium(9, np.ones(n), np.zeros(n), np.zeros(n), None, prec=64))
    y = (np.arange(ny) + 0.5) / ny
    T = np.repeat(1.0 - y, nx)
    o.set_thermal_state(np.outer(np.array([2.0, 1.0, 1.0, 1.0, 1.0]) / 6.0, T))
    o.step(500)
    assert np.abs(o.temperature() - T).max() < 1e-9
    assert np.abs(o.macro()["uy"]).max() < 1e-9


def test_thermal_energy_follows_wall_flux():
    """With both walls at the reference temperature and a uniform start at it, nothing moves."""
    nx, ny = 16, 8
    o = oracle.OracleGrid(9, nx, ny, 1, 64)
    o.configure(collision=0, tau=0.7, thermal=1, tau_t=0.8, t_ref=0.3, beta_g=1e-3, t_south=0.3, t_north=0.3)
    o.set_cell_types(np.zeros(nx * ny, np.uint8))
    n = nx * ny
    o.set_state(oracle.equilibrium(9, np.ones(n), np.zeros(n), np.zeros(n), None, prec=64))
    o.set_thermal_state(np.outer(np.array([2.0, 1.0, 1.0, 1.0, 1.0]) / 6.0, np.full(n, 0.3)))
    o.step(200)
    assert np.abs(o.temperature() - 0.3).max() < 1e-12
    assert np.abs(o.macro()["ux"]).max() < 1e-12
