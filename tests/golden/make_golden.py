#!/usr/bin/env python3
"""Generate the golden fixtures in this directory from the reference itself.

Runs the reference's own host classes and its ISPC kernels (mechanically
translated to C++ by oracle/build_ref.py, as ISPC is not installed here) on
small seeded inputs and stores inputs and outputs as .npz files. The GPU tests
compare against these files, so they need neither the reference sources nor
its build on the GPU machine.

    python tests/golden/make_golden.py     (needs the reference sources)
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from wake_b200 import workloads as W  # noqa: E402

OUT = Path(__file__).resolve().parent


def a(x):
    return None if x is None else x.ctypes.data


def save(name, **arrays):
    np.savez_compressed(OUT / f"{name}.npz", **arrays)
    print(f"wrote {name}.npz ({(OUT / f'{name}.npz').stat().st_size} bytes)")


def cylinder_cases(R):
    for coll, tag in ((0, "bgk"), (1, "trt"), (2, "mrt")):
        c = W.cylinder_channel(nx=64, ny=32, diameter=8, cx=16, cy=16, tau=0.56, collision=coll)
        g = oracle.RefGrid2D(c.nx, c.ny, c.tau)
        g.init_fields(c.rho, c.ux, c.uy)
        R.ref2d_set_inflow_west(g._h, 0.05, 0.0)
        R.ref2d_set_outflow_east(g._h, 1.0)
        for x in range(c.nx):
            R.ref2d_set_cell_type(g._h, x, 0, 1)
            R.ref2d_set_cell_type(g._h, x, c.ny - 1, 1)
        R.ref2d_set_solid_circle(g._h, 16.0, 16.0, 4.0)
        assert (g.cell_types() == c.types).all()
        f0 = g.f()
        hist = g.step_forces(200, coll, 16.0, 16.0, 12.0)
        m = g.macro()
        save(f"cyl2d_{tag}", f0=f0, types=c.types, steps=np.int32(200), tau=np.float32(c.tau), collision=np.int32(coll),
             rho=m["rho"], ux=m["ux"], uy=m["uy"], speed=m["speed"], forces=hist, f_end=g.f())


def cavity_case(R):
    n = 32
    g = oracle.RefGrid2D(n, n, 0.6)
    g.init_fields(np.ones(n * n, np.float32), np.zeros(n * n, np.float32), np.zeros(n * n, np.float32))
    for x in range(n):
        R.ref2d_set_cell_type(g._h, x, 0, 1)
    for y in range(n):
        R.ref2d_set_cell_type(g._h, 0, y, 1)
        R.ref2d_set_cell_type(g._h, n - 1, y, 1)
    R.ref2d_set_moving_wall_north(g._h, 0.1)
    f0 = g.f()
    # the reference's lid row is itself collided and streamed as fluid and pulls the wall
    # momentum from its lid neighbours; the cavity diverges after ~120 steps, so stop at 80
    g.step(80, 2)
    m = g.macro()
    save("cavity2d_mrt", f0=f0, types=g.cell_types(), steps=np.int32(80), tau=np.float32(0.6), lid=np.float32(0.1),
         rho=m["rho"], ux=m["ux"], uy=m["uy"])


def poiseuille_case(R):
    # body-force channel (tests/validation/test_poiseuille_convergence.cpp:12-31), TRT
    nx, ny = 8, 33
    g = oracle.RefGrid2D(nx, ny, 0.8)
    for x in range(nx):
        R.ref2d_set_cell_type(g._h, x, 0, 1)
        R.ref2d_set_cell_type(g._h, x, ny - 1, 1)
    f0 = g.f()
    g.step(500, 1, 1e-4, 0.0)
    m = g.macro()
    save("poiseuille2d_trt", f0=f0, types=g.cell_types(), steps=np.int32(500), tau=np.float32(0.8), gx=np.float32(1e-4),
         rho=m["rho"], ux=m["ux"], uy=m["uy"])


def sphere_cases(R):
    for coll, tag in ((0, "bgk"), (1, "trt"), (2, "mrt")):
        c = W.sphere_channel(nx=24, ny=16, nz=16, radius=4.0, center=(8.0, 8.0, 8.0), tau=0.6, collision=coll,
                             reference_variant=True)
        g = oracle.RefGrid3D(c.nx, c.ny, c.nz, c.tau)
        g.init_fields(c.rho, c.ux, c.uy, c.uz)
        R.ref3d_set_periodic(g._h, 1)
        R.ref3d_set_solid_sphere(g._h, 8.0, 8.0, 8.0, 4.0)
        R.ref3d_build_curved_sphere_links(g._h, 8.0, 8.0, 8.0, 4.0)
        assert (g.cell_types() == c.types).all()
        idx, q, d = g.links()
        f0 = g.f()
        hist = g.step_forces(60, coll, (8.0, 8.0, 8.0), 8.0)
        m = g.macro()
        save(f"sphere3d_{tag}", f0_node=f0[:, 0].copy(), types=c.types, links_idx=idx, links_q=q, links_delta=d,
             steps=np.int32(60), tau=np.float32(c.tau), collision=np.int32(coll), rho=m["rho"], ux=m["ux"],
             uy=m["uy"], uz=m["uz"], forces=hist)


def tgv_case(R):
    c = W.taylor_green(L=12, u0=0.04, tau=0.56, q=19, collision=2)
    g = oracle.RefGrid3D(c.nx, c.ny, c.nz, c.tau)
    R.ref3d_set_periodic(g._h, 1)
    g.init_fields(c.rho, c.ux, c.uy, c.uz)
    f0 = g.f()
    g.step(30, 2)
    m = g.macro()
    save("tgv3d_mrt", f0=f0, steps=np.int32(30), tau=np.float32(c.tau), rho=m["rho"], ux=m["ux"], uy=m["uy"],
         uz=m["uz"])


def percall_cases(R):
    """Inputs and outputs of single kernel calls (per-call drop-in parity)."""
    F = np.float32
    rng = lambda seed, n: W.uniform24(seed, n)  # noqa: E731
    res = {}
    # collisions
    for Q, pref in ((9, "d2q9"), (19, "d3q19"), (27, "d3q27")):
        count = 96
        w = oracle.equilibrium(Q, np.ones(1), np.zeros(1), np.zeros(1), np.zeros(1) if Q != 9 else None)[:, 0]
        f = (w[:, None] * (1.0 + 0.2 * (rng(W.BASE_SEED + Q, Q * count).reshape(Q, count) - 0.5))).astype(F)
        ct = np.zeros(count, np.uint8)
        ct[::7] = 1
        res[f"{pref}_f"] = f
        res[f"{pref}_ct"] = ct
        models = {9: [("bgk", (0.7,)), ("trt", (0.7, 1.2)), ("mrt", (0.7, 1.6))],
                  19: [("bgk", (0.75,)), ("trt", (0.75, 1.3)), ("mrt", (0.75, 1.2))],
                  27: [("collide", (0.75, 1.3))]}[Q]
        for name, taus in models:
            out = np.zeros_like(f)
            rho, ux, uy, uz = (np.zeros(count, F) for _ in range(4))
            fn = getattr(R, f"{pref}_collide_{name}" if Q != 27 else "d3q27_collide")
            gvec = (1e-5, -2e-5) if Q == 9 else (1e-5, -2e-5, 3e-5)
            if Q == 9:
                fn.argtypes = [C.c_void_p] * 6 + [C.c_float] * (len(taus) + 2) + [C.c_int]
                fn(a(f), a(out), a(ct), a(rho), a(ux), a(uy), *taus, *gvec, count)
            else:
                fn.argtypes = [C.c_void_p] * 7 + [C.c_float] * (len(taus) + 3) + [C.c_int]
                fn(a(f), a(out), a(ct), a(rho), a(ux), a(uy), a(uz), *taus, *gvec, count)
            key = f"{pref}_{name}"
            res[f"{key}_out"], res[f"{key}_rho"], res[f"{key}_ux"], res[f"{key}_uy"] = out, rho, ux, uy
            if Q != 9:
                res[f"{key}_uz"] = uz
    # streaming + Zou-He + moments + LES + MEM on a small 2D channel state
    nx, ny = 20, 12
    n = nx * ny
    w9 = oracle.equilibrium(9, np.ones(1), np.zeros(1), np.zeros(1))[:, 0]
    f = (w9[:, None] * (1.0 + 0.1 * (rng(W.BASE_SEED + 100, 9 * n).reshape(9, n) - 0.5))).astype(F)
    ct = np.zeros((ny, nx), np.uint8)
    ct[0, :] = 1
    ct[ny - 1, :] = 6
    ct[5:7, 8:10] = 1
    ct = ct.ravel()
    res["s2_f"], res["s2_ct"] = f, ct
    dst = np.zeros_like(f)
    R.d2q9_stream_with_boundaries.argtypes = [C.c_void_p] * 3 + [C.c_int] * 2 + [C.c_float] * 2
    R.d2q9_stream_with_boundaries(a(f), a(dst), a(ct), nx, ny, 0.08, 0.0)
    res["s2_stream"] = dst.copy()
    per = np.zeros_like(f)
    R.d2q9_stream_periodic.argtypes = [C.c_void_p] * 2 + [C.c_int] * 2
    R.d2q9_stream_periodic(a(f), a(per), nx, ny)
    res["s2_periodic"] = per
    fz = f.copy()
    rho, ux, uy = (np.zeros(n, F) for _ in range(3))
    R.d2q9_apply_zou_he_inflow_west.argtypes = [C.c_void_p] * 4 + [C.c_float] * 2 + [C.c_int] * 2
    R.d2q9_apply_zou_he_inflow_west(a(fz), a(rho), a(ux), a(uy), 0.05, 0.01, nx, ny)
    R.d2q9_apply_zou_he_outflow_east.argtypes = [C.c_void_p] * 4 + [C.c_float] + [C.c_int] * 2
    R.d2q9_apply_zou_he_outflow_east(a(fz), a(rho), a(ux), a(uy), 1.01, nx, ny)
    res["s2_zh_f"], res["s2_zh_rho"], res["s2_zh_ux"], res["s2_zh_uy"] = fz, rho, ux, uy
    rho, ux, uy, sp = (np.zeros(n, F) for _ in range(4))
    R.d2q9_compute_macroscopic_moments_forced.argtypes = [C.c_void_p] * 4 + [C.c_float] * 2 + [C.c_int]
    R.d2q9_compute_macroscopic_moments_forced(a(f), a(rho), a(ux), a(uy), 1e-4, -2e-4, n)
    R.d2q9_compute_velocity_magnitude.argtypes = [C.c_void_p] * 3 + [C.c_int]
    R.d2q9_compute_velocity_magnitude(a(ux), a(uy), a(sp), n)
    res["s2_mf_rho"], res["s2_mf_ux"], res["s2_mf_uy"], res["s2_speed"] = rho, ux, uy, sp
    tau_eff = np.zeros(n, F)
    R.d2q9_compute_smagorinsky_tau.argtypes = [C.c_void_p] * 5 + [C.c_float] * 2 + [C.c_int]
    R.d2q9_compute_smagorinsky_tau(a(f), a(rho), a(ux), a(uy), a(tau_eff), 0.52, 0.17, n)
    res["s2_tau_eff"] = tau_eff
    fx, fy, tz = C.c_float(), C.c_float(), C.c_float()
    R.d2q9_compute_momentum_exchange_forces.argtypes = [C.c_void_p] * 2 + [C.c_int] * 2 + [C.c_float] * 3 + [C.c_void_p] * 3
    R.d2q9_compute_momentum_exchange_forces(a(f), a(ct), nx, ny, 8.5, 5.5, 4.0, C.byref(fx), C.byref(fy), C.byref(tz))
    res["s2_mem"] = np.array([fx.value, fy.value, tz.value], F)
    # 3D streaming with walls + BFL + MEM
    nx, ny, nz = 10, 8, 6
    n = nx * ny * nz
    w19 = oracle.equilibrium(19, np.ones(1), np.zeros(1), np.zeros(1), np.zeros(1))[:, 0]
    f = (w19[:, None] * (1.0 + 0.1 * (rng(W.BASE_SEED + 200, 19 * n).reshape(19, n) - 0.5))).astype(F)
    ct = np.zeros((nz, ny, nx), np.uint8)
    ct[2:4, 3:5, 4:6] = 1
    ct[:, ny - 1, :] = 6
    ct = ct.ravel()
    res["s3_f"], res["s3_ct"] = f, ct
    dst = np.zeros_like(f)
    R.d3q19_stream_with_boundaries.argtypes = [C.c_void_p] * 3 + [C.c_int] * 3 + [C.c_float] * 3
    R.d3q19_stream_with_boundaries(a(f), a(dst), a(ct), nx, ny, nz, 0.05, 0.0, 0.02)
    res["s3_stream"] = dst.copy()
    per = np.zeros_like(f)
    R.d3q19_stream_periodic.argtypes = [C.c_void_p] * 2 + [C.c_int] * 3
    R.d3q19_stream_periodic(a(f), a(per), nx, ny, nz)
    res["s3_periodic"] = per
    links = [(i, q) for i in range(n) if ct[i] == 0 for q in range(1, 19)]
    xs = lambda i: (i % nx, (i // nx) % ny, i // (nx * ny))  # noqa: E731
    lat = np.array([[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1], [1, 1, 0],
                    [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1], [-1, 0, -1], [0, 1, 1],
                    [0, -1, 1], [0, 1, -1], [0, -1, -1]])
    sel = []
    for i, q in links:
        x, y, z = xs(i)
        xn, yn, zn = (x + lat[q, 0]) % nx, y + lat[q, 1], z + lat[q, 2]
        if 0 <= yn < ny and 0 <= zn < nz and ct[(zn * ny + yn) * nx + xn] == 1:
            sel.append((i, q))
    idx = np.array([s[0] for s in sel], np.int32)
    qd = np.array([s[1] for s in sel], np.int32)
    nl = len(idx)
    delta = (0.05 + 0.9 * rng(W.BASE_SEED + 300, nl)).astype(F)
    uwx, uwy, uwz = (0.01 * (rng(W.BASE_SEED + 301, nl) - 0.5)).astype(F), np.zeros(nl, F), np.zeros(nl, F)
    fb = dst.copy()
    R.d3q19_apply_curved_bfl.argtypes = [C.c_void_p] * 8 + [C.c_int] * 4
    R.d3q19_apply_curved_bfl(a(fb), a(f), a(idx), a(qd), a(delta), a(uwx), a(uwy), a(uwz), nx, ny, nz, nl)
    res.update(s3_bfl_idx=idx, s3_bfl_q=qd, s3_bfl_delta=delta, s3_bfl_uwx=uwx, s3_bfl_out=fb)
    fx, fy, fz = C.c_float(), C.c_float(), C.c_float()
    R.d3q19_compute_momentum_exchange_forces.argtypes = [C.c_void_p] * 2 + [C.c_int] * 3 + [C.c_float] * 4 + [C.c_void_p] * 3
    R.d3q19_compute_momentum_exchange_forces(a(f), a(ct), nx, ny, nz, 4.5, 3.5, 2.5, 0.0, C.byref(fx), C.byref(fy),
                                             C.byref(fz))
    res["s3_mem"] = np.array([fx.value, fy.value, fz.value], F)
    rho, ux, uy, uz, tau_eff = (np.zeros(n, F) for _ in range(5))
    R.d3q19_compute_macroscopic_moments.argtypes = [C.c_void_p] * 5 + [C.c_int]
    R.d3q19_compute_macroscopic_moments(a(f), a(rho), a(ux), a(uy), a(uz), n)
    R.d3q19_compute_smagorinsky_tau.argtypes = [C.c_void_p] * 6 + [C.c_float] * 2 + [C.c_int]
    R.d3q19_compute_smagorinsky_tau(a(f), a(rho), a(ux), a(uy), a(uz), a(tau_eff), 0.52, 0.17, n)
    res.update(s3_rho=rho, s3_ux=ux, s3_uy=uy, s3_uz=uz, s3_tau_eff=tau_eff)
    # D3Q27 periodic stream
    f27 = rng(W.BASE_SEED + 400, 27 * n).reshape(27, n).astype(F)
    per = np.zeros_like(f27)
    R.d3q27_stream_periodic.argtypes = [C.c_void_p] * 2 + [C.c_int] * 3
    R.d3q27_stream_periodic(a(f27), a(per), nx, ny, nz)
    res.update(s27_f=f27, s27_periodic=per)
    # thermal
    nx, ny = 12, 8
    n = nx * ny
    gi = (w9[:, None] * (0.5 + rng(W.BASE_SEED + 500, 9 * n).reshape(9, n))).astype(F)
    ctt = np.zeros(n, np.uint8)
    ctt[5] = 1
    ux = (0.02 * (rng(W.BASE_SEED + 501, n) - 0.5)).astype(F)
    uy = (0.02 * (rng(W.BASE_SEED + 502, n) - 0.5)).astype(F)
    go = np.zeros_like(gi)
    T = np.zeros(n, F)
    R.thermal_collide_d2q9.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_int]
    R.thermal_collide_d2q9(a(gi), a(go), a(ctt), a(ux), a(uy), a(T), 0.7, n)
    gw = go.copy()
    R.thermal_apply_isothermal_wall.argtypes = [C.c_void_p] + [C.c_int] * 3 + [C.c_float]
    R.thermal_apply_isothermal_wall(a(gw), nx, ny, 0, 1.0)
    gy = np.full(n, 1e-5, F)
    R.thermal_compute_buoyancy_force_2d.argtypes = [C.c_void_p] * 2 + [C.c_float] * 3 + [C.c_int]
    R.thermal_compute_buoyancy_force_2d(a(T), a(gy), 0.5, 0.01, 0.1, n)
    res.update(th_g=gi, th_ct=ctt, th_ux=ux, th_uy=uy, th_out=go, th_T=T, th_wall=gw, th_gy=gy)
    save("percall", **res)


def c1_case(R, steps=20000):
    """The full D2Q9 BGK cylinder channel (400x160, D = 20 at (80, 80), tau = 0.56, seeded 1e-4
    noise): the reference's own 20,000 steps with momentum exchange (r_max = 1.5 D) every step,
    as KarmanVortexScenario runs it (src/scenarios/karman_vortex.cpp:62-124). Stores the force
    history and the reference's Strouhal frequency of its lift (StrouhalAnalyzer, first 4096
    samples)."""
    c = W.cylinder_channel()
    g = oracle.RefGrid2D(c.nx, c.ny, c.tau)
    g.init_fields(c.rho, c.ux, c.uy)
    R.ref2d_set_inflow_west(g._h, 0.05, 0.0)
    R.ref2d_set_outflow_east(g._h, 1.0)
    for x in range(c.nx):
        R.ref2d_set_cell_type(g._h, x, 0, 1)
        R.ref2d_set_cell_type(g._h, x, c.ny - 1, 1)
    R.ref2d_set_solid_circle(g._h, 80.0, 80.0, 10.0)
    assert (g.cell_types() == c.types).all()
    f0 = g.f()
    hist = g.step_forces(steps, 0, 80.0, 80.0, 30.0)
    cl = (hist[:, 1] / (0.5 * 0.05 ** 2 * 20.0)).astype(np.float32)
    f_ref = R.ref_strouhal_frequency(a(cl), len(cl), 1.0)
    # the same run in the FP64 oracle, the yardstick for the FP32 drift of either implementation
    o = oracle.OracleGrid(9, c.nx, c.ny, 1, 64)
    o.configure(collision=0, tau=c.tau, inflow=1, outflow=1, u_in=(0.05, 0.0, 0.0), rho_out=1.0, mem=1,
                center=(80.0, 80.0, 0.0), r_max=30.0)
    o.set_cell_types(c.types)
    o.set_state(f0)
    h64 = o.step(steps, forces=True)
    # Fx, Fy per step; the FP64 history rounded to float32 (6e-8 relative, far below its 5e-5 gap to FP32)
    save("c1_cyl2d_bgk", forces=hist[:, :2].astype(np.float32), forces_fp64=h64[:, :2].astype(np.float32),
         steps=np.int32(steps),
         tau=np.float32(c.tau), strouhal_freq=np.float32(f_ref), f0_sum=np.float64(f0.astype(np.float64).sum()))


def c2_case(R, steps=2000):
    """The D3Q19 sphere channel at full size (256x128x128, sphere R = 12 at (64, 64, 64), TRT with
    Lambda = 1/4, tau0 = 0.52, 2000 steps) in the form the reference can run: x-periodic, y/z
    half-way walls, no Zou-He, LES computed but not applied. The reference's own run gives the
    per-step force history and the moments on two planes through the sphere (z = 64 and y = 64,
    every other node in each direction);
    the FP64 oracle runs the same case from the same populations and links, and its results are
    stored rounded to float32 (6e-8 relative, far below their 1e-5 gap to FP32)."""
    c = W.sphere_channel(reference_variant=True, collision=1, les=False)
    cx, cy, cz, r = c.sphere
    g = oracle.RefGrid3D(c.nx, c.ny, c.nz, c.tau)
    g.init_fields(c.rho, c.ux, c.uy, c.uz)
    R.ref3d_set_periodic(g._h, 1)
    R.ref3d_set_solid_sphere(g._h, cx, cy, cz, r)
    R.ref3d_build_curved_sphere_links(g._h, cx, cy, cz, r)
    assert (g.cell_types() == c.types).all()
    idx, q, d = g.links()
    f0 = g.f()
    hist = g.step_forces(steps, 1, (cx, cy, cz), c.mem[3])
    m = g.macro()

    def planes(fields):
        out = {}
        for k in ("rho", "ux", "uy", "uz"):
            a = np.asarray(fields[k]).reshape(c.nz, c.ny, c.nx)
            out[f"{k}_z64"] = np.ascontiguousarray(a[64][::2, ::2]).astype(np.float32)  # every other node
            out[f"{k}_y64"] = np.ascontiguousarray(a[:, 64, :][::2, ::2]).astype(np.float32)
        return out

    o = oracle.OracleGrid(19, c.nx, c.ny, c.nz, 64)
    o.configure(collision=1, tau=c.tau, les=0, periodic_y=0, periodic_z=0, mem=1, center=(cx, cy, cz),
                r_max=c.mem[3])
    o.set_cell_types(c.types)
    o.set_state(f0)
    o.set_links(idx, q, d)
    h64 = o.step(steps, forces=True)
    m64 = o.macro()
    ref_planes, o_planes = planes(m), planes(m64)
    save("c2_sphere3d_trt", steps=np.int32(steps), tau=np.float32(c.tau), forces=hist.astype(np.float32),
         forces_fp64=h64.astype(np.float32), n_links=np.int32(len(idx)),
         **{f"ref_{k}": v for k, v in ref_planes.items()}, **{f"fp64_{k}": v for k, v in o_planes.items()})


C3_EDGE, C3_EVERY, C3_STEPS, C3_SUB = 96, 500, 5000, 3


def c3_case(edge=C3_EDGE, steps=C3_STEPS, every=C3_EVERY, sub=C3_SUB):
    """The C3 Taylor-Green vortex (D3Q27 MRT, u0 = 0.04, tau = 0.51, 5000 steps) on an edge^3
    periodic cube, in the FP64 oracle only: the reference has no D3Q27 MRT, so FP64 is the
    yardstick of the FP32 / FP16 / BF16 storages. The start is the equilibrium of the float32
    fields, rounded to float32 (the GPU's initial state). Every `every` steps: the FP64 kinetic
    energy sum(rho |u|^2 / 2) over all nodes and the velocity on every `sub`-th node in each
    direction, rounded to float32 (6e-8 relative, far below the storage errors measured)."""
    c = W.taylor_green(L=edge, u0=0.04, tau=0.51, q=27, collision=2)
    o = oracle.OracleGrid(27, edge, edge, edge, 64)
    o.configure(collision=2, tau=c.tau, periodic_y=1, periodic_z=1)
    o.set_cell_types(c.types)
    o.set_state(oracle.equilibrium(27, c.rho, c.ux, c.uy, c.uz, prec=32).astype(np.float32))
    # initial kinetic energy from the initial fields (the equilibrium's moments reproduce them to
    # float32 rounding); later entries from the oracle's moments after each checkpoint's step
    ke = [0.5 * float((c.rho.astype(np.float64) * (c.ux.astype(np.float64) ** 2 + c.uy.astype(np.float64) ** 2 +
                                                     c.uz.astype(np.float64) ** 2)).sum())]
    u = []
    for k in range(steps // every):
        o.step(every)
        m = o.macro()
        ke.append(0.5 * float((m["rho"] * m["speed"] ** 2).sum()))
        u.append(np.stack([m[a].reshape(edge, edge, edge)[::sub, ::sub, ::sub].astype(np.float32)
                           for a in ("ux", "uy", "uz")]))
        print(f"c3: step {(k + 1) * every} KE/KE0 {ke[-1] / ke[0]:.6f}", flush=True)
    save(f"c3_tgv{edge}_mrt_fp64", edge=np.int32(edge), steps=np.int32(steps), every=np.int32(every),
         sub=np.int32(sub), tau=np.float32(c.tau), u0=np.float32(0.04), ke=np.array(ke, np.float64),
         u=np.stack(u))


def diag_cases(R, steps=200):
    """The reference's global diagnostics (compute_total_mass, compute_total_kinetic_energy,
    compute_max_speed: serial float sums over Fluid cells only, src/grid/lattice_grid_2d.cpp:267-295,
    src/grid/lattice_grid_3d.cpp:382-410) after `steps` steps of a cylinder channel that holds
    Solid, Inflow and Outflow cells (TRT, the cyl2d set-up) and of a sphere with curved links
    (TRT, the sphere3d set-up). Also stored: the same sums in FP64 over the reference's own
    fields, over Fluid cells and over every non-solid cell."""
    out = {}
    c = W.cylinder_channel(nx=64, ny=32, diameter=8, cx=16, cy=16, tau=0.56, collision=1)
    g = oracle.RefGrid2D(c.nx, c.ny, c.tau)
    g.init_fields(c.rho, c.ux, c.uy)
    R.ref2d_set_inflow_west(g._h, 0.05, 0.0)
    R.ref2d_set_outflow_east(g._h, 1.0)
    for x in range(c.nx):
        R.ref2d_set_cell_type(g._h, x, 0, 1)
        R.ref2d_set_cell_type(g._h, x, c.ny - 1, 1)
    R.ref2d_set_solid_circle(g._h, 16.0, 16.0, 4.0)
    t = g.cell_types()
    out.update(d2_types=t, d2_f0=g.f(), d2_steps=np.int32(steps), d2_tau=np.float32(c.tau))
    g.step(steps, 1)
    m = g.macro()
    out.update(d2_mass=np.float32(R.ref2d_total_mass(g._h)), d2_ke=np.float32(R.ref2d_total_ke(g._h)),
               d2_vmax=np.float32(R.ref2d_max_speed(g._h)))
    fluid, open_ = t == 0, t != 1
    rho, sp = m["rho"].astype(np.float64), m["speed"].astype(np.float64)
    out.update(d2_mass64=rho[fluid].sum(), d2_ke64=(0.5 * rho * sp * sp)[fluid].sum(),
               d2_mass64_open=rho[open_].sum(), d2_ke64_open=(0.5 * rho * sp * sp)[open_].sum())
    nx, ny, nz = 24, 16, 16
    g3 = oracle.RefGrid3D(nx, ny, nz, 0.56)
    n = nx * ny * nz
    noise = W.uniform24(W.BASE_SEED + 600, 3 * n).reshape(3, n)
    g3.init_fields(np.ones(n, np.float32), (0.04 + 0.01 * (noise[0] - 0.5)).astype(np.float32),
                   (0.01 * (noise[1] - 0.5)).astype(np.float32), (0.01 * (noise[2] - 0.5)).astype(np.float32))
    R.ref3d_set_solid_sphere(g3._h, 8.0, 8.0, 8.0, 4.0)
    R.ref3d_build_curved_sphere_links(g3._h, 8.0, 8.0, 8.0, 4.0)
    t3 = g3.cell_types()
    out.update(d3_types=t3, d3_f0_sum=np.float64(g3.f().astype(np.float64).sum()), d3_steps=np.int32(steps))
    R.ref3d_step(g3._h, 1, 0.0, 0.0, 0.0, 0, 0.14, steps)
    m3 = g3.macro()
    out.update(d3_mass=np.float32(R.ref3d_total_mass(g3._h)), d3_ke=np.float32(R.ref3d_total_ke(g3._h)),
               d3_vmax=np.float32(R.ref3d_max_speed(g3._h)))
    fl3 = t3 == 0
    rho3, sp3 = m3["rho"].astype(np.float64), m3["speed"].astype(np.float64)
    out.update(d3_mass64=rho3[fl3].sum(), d3_ke64=(0.5 * rho3 * sp3 * sp3)[fl3].sum())
    save("diag", **out)


def kat_cases(R):
    # Strouhal FFT KAT (tests/unit/test_forces_momentum_exchange.cpp:71-91)
    t = np.arange(512, dtype=np.float32)
    sig = (np.float32(0.35) * np.sin(np.float32(6.2831855) * np.float32(0.025) * t) +
           np.float32(0.02) * np.cos(np.float32(6.2831855) * np.float32(0.1) * t)).astype(np.float32)
    f = R.ref_strouhal_frequency(a(sig), len(sig), 1.0)
    save("kat", strouhal_signal=sig, strouhal_freq=np.float32(f))


def main():
    R = oracle.ref()
    if R is None:
        raise SystemExit("reference library unavailable: run oracle/build_ref.py where the reference sources exist")
    cylinder_cases(R)
    cavity_case(R)
    poiseuille_case(R)
    sphere_cases(R)
    tgv_case(R)
    percall_cases(R)
    kat_cases(R)
    diag_cases(R)
    c1_case(R)
    c2_case(R)


if __name__ == "__main__":
    if "--c1" in sys.argv:  # only the long C1 run
        c1_case(oracle.ref())
    elif "--c2" in sys.argv:  # only the full-size C2 run (about an hour on one core)
        c2_case(oracle.ref())
    elif "--diag" in sys.argv:  # only the diagnostics fixture
        diag_cases(oracle.ref())
    elif "--c3" in sys.argv:  # only the FP64 Taylor-Green run (oracle only; about 30 min on 8 threads)
        c3_case()
    else:
        main()
