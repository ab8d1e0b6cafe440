"""Seeded synthetic workloads of the benchmark configurations.

All random numbers come from SplitMix64 (Steele, Lea & Flood, "Fast splittable
pseudorandom number generators", OOPSLA 2014), counter-based so any slice can
be regenerated, turned into 24-bit uniform floats. Base seed 20261203; domain
``d`` of a workload uses seed base + d. The same arrays feed the GPU engine,
the CPU oracle and the reference, so all three start from identical bytes.

Scenario layouts follow the reference scenarios they are modelled on:
cylinder channel = KarmanVortexScenario::setup (src/scenarios/karman_vortex.cpp:62-88),
sphere = Sphere3DWakeScenario::setup (src/scenarios/sphere_3d_wake.cpp:64-78),
Taylor-Green = tests/validation/test_taylor_green_decay.cpp:22-33.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

BASE_SEED = 20261203
_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

FLUID, SOLID, INFLOW, OUTFLOW, MOVING_WALL = 0, 1, 2, 3, 6


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """Outputs offset+1 .. offset+n of the SplitMix64 stream of ``seed``."""
    with np.errstate(over="ignore"):
        i = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed % (1 << 64)) + i * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform24(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n floats in [0, 1) with 24 random bits each."""
    return (splitmix64(seed, n, offset) >> np.uint64(40)).astype(np.float32) * np.float32(2.0**-24)


@dataclass
class Case:
    """One lattice with geometry, initial state and run parameters.

    ``init`` describes the initial velocity field, from which the initial
    populations are the equilibrium (rho, u):
      ("uniform", rho, (ux, uy, uz))
      ("noise", rho, (ux, uy, uz), amplitude, seed, offset): u_a + amplitude * (2 r - 1)
          with r = uniform24 output offset + a*N + i of the seed's stream (component a, node i)
      ("fields", rho[N], ux[N], uy[N], uz[N])
    The ``rho`` / ``ux`` / ``uy`` / ``uz`` arrays are built on first use only;
    ``build_grid`` initialises uniform and noisy states on the device.
    """

    q: int
    nx: int
    ny: int
    nz: int
    types: np.ndarray | None   # uint8 [N]; None: geometry set on the device (extra["device_sphere"])
    init: tuple
    tau: float
    collision: int
    les: bool = False
    cs_smag: float = 0.14
    inflow: tuple | None = None      # (ux, uy, uz) Zou-He inlet
    outflow: float | None = None     # rho_out
    periodic_y: bool = False
    periodic_z: bool = False
    sphere: tuple | None = None      # (cx, cy, cz, R) for curved links
    mem: tuple | None = None         # (cx, cy, cz, r_max)
    ref_area: float = 1.0            # force coefficient area (D in 2D, pi R^2 in 3D)
    u_ref: float = 0.05
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.nx * self.ny * self.nz

    def fields(self) -> tuple:
        """(rho, ux, uy, uz) float32 arrays of the initial state."""
        cached = self.extra.get("_fields")
        if cached is not None:
            return cached
        n, kind = self.n, self.init[0]
        if kind == "fields":
            out = tuple(np.ascontiguousarray(a, np.float32).ravel() for a in self.init[1:5])
        else:
            rho = np.full(n, self.init[1], np.float32)
            u = [np.full(n, np.float32(c), np.float32) for c in self.init[2]]
            if kind == "noise":
                amp, seed, off = self.init[3], self.init[4], self.init[5]
                dims = 3 if self.q != 9 else 2
                r = uniform24(seed, dims * n, off)
                for a in range(dims):
                    u[a] = (np.float32(self.init[2][a]) + np.float32(amp) *
                            (np.float32(2.0) * r[a * n:(a + 1) * n] - np.float32(1.0))).astype(np.float32)
            out = (rho, u[0], u[1], u[2])
        self.extra["_fields"] = out
        return out

    @property
    def rho(self) -> np.ndarray:
        return self.fields()[0]

    @property
    def ux(self) -> np.ndarray:
        return self.fields()[1]

    @property
    def uy(self) -> np.ndarray:
        return self.fields()[2]

    @property
    def uz(self) -> np.ndarray:
        return self.fields()[3]


def cylinder_channel(nx=400, ny=160, diameter=20.0, cx=80.0, cy=80.0, u_in=0.05, tau=0.56, collision=0,
                     noise=1e-4, seed=BASE_SEED) -> Case:
    """2D channel: Zou-He inlet/outlet, solid rows y=0 and y=ny-1, solid disk.

    Cell types are set in the order of KarmanVortexScenario::setup: inlet
    column, outlet column, wall rows, then the disk (LatticeGrid2D::set_solid_circle).
    """
    t = np.zeros((ny, nx), np.uint8)
    t[:, 0] = INFLOW
    t[:, nx - 1] = OUTFLOW
    t[0, :] = SOLID
    t[ny - 1, :] = SOLID
    _rasterize_circle(t, cx, cy, diameter * 0.5)
    return Case(q=9, nx=nx, ny=ny, nz=1, types=t.ravel(), init=("noise", 1.0, (u_in, 0.0, 0.0), noise, seed, 0),
                tau=tau, collision=collision,
                inflow=(u_in, 0.0, 0.0), outflow=1.0, mem=(cx, cy, 0.0, 1.5 * diameter), ref_area=diameter,
                u_ref=u_in)


def _rasterize_circle(t: np.ndarray, cx: float, cy: float, radius: float) -> None:
    """LatticeGrid2D::set_solid_circle (src/grid/lattice_grid_2d.cpp:143-158) in float32."""
    ny, nx = t.shape
    f32 = np.float32
    r_sq = f32(radius) * f32(radius)
    min_x = max(0, int(f32(cx) - f32(radius) - f32(1)))
    max_x = min(nx - 1, int(f32(cx) + f32(radius) + f32(1)))
    min_y = max(0, int(f32(cy) - f32(radius) - f32(1)))
    max_y = min(ny - 1, int(f32(cy) + f32(radius) + f32(1)))
    for y in range(min_y, max_y + 1):
        for x in range(min_x, max_x + 1):
            dx = f32(x) - f32(cx)
            dy = f32(y) - f32(cy)
            if dx * dx + dy * dy <= r_sq:
                t[y, x] = SOLID


def _rasterize_ellipse(t: np.ndarray, cx: float, cy: float, a: float, b: float, angle: float) -> None:
    """Rotated ellipse in float32, the rule of wake_grid_set_solid_ellipse (cell centres
    at integer coordinates; cos/sin evaluated in double and rounded to float)."""
    ny, nx = t.shape
    f32 = np.float32
    r = max(f32(a), f32(b))
    min_x = max(0, int(f32(cx) - r - f32(1)))
    max_x = min(nx - 1, int(f32(cx) + r + f32(1)))
    min_y = max(0, int(f32(cy) - r - f32(1)))
    max_y = min(ny - 1, int(f32(cy) + r + f32(1)))
    ang = float(f32(angle))
    c, s = f32(math.cos(ang)), f32(math.sin(ang))
    inv_a2 = f32(1.0) / (f32(a) * f32(a))
    inv_b2 = f32(1.0) / (f32(b) * f32(b))
    ys = np.arange(min_y, max_y + 1)
    xs = np.arange(min_x, max_x + 1)
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    dx = X.astype(f32) - f32(cx)
    dy = Y.astype(f32) - f32(cy)
    u = dx * c + dy * s
    v = -dx * s + dy * c
    inside = (u * u * inv_a2 + v * v * inv_b2) <= f32(1.0)
    sub = t[min_y:max_y + 1, min_x:max_x + 1]
    sub[inside] = SOLID


def ellipse_channel(nx: int, ny: int, a: float, b: float, angle_deg: float, reynolds: float, u_in: float = 0.05,
                    collision: int = 1, les: bool = True, cs_smag: float = 0.17, noise: float = 1e-4,
                    seed: int = BASE_SEED, noise_offset: int = 0) -> Case:
    """2D channel around a rotated ellipse (the batched sweep's domain).

    Layout as cylinder_channel: Zou-He inlet u_in on x = 0, outlet rho = 1 on
    x = nx-1, solid rows y = 0 and y = ny-1, obstacle centred at (nx/5, ny/2).
    tau from nu = u_in * 2a / Re (chord 2a). Momentum exchange within 1.5 chords.
    The Smagorinsky model (Cs = 0.17, as the sphere channel) is on by default: at
    the sweep's smallest chords tau comes within 0.004 of 1/2 and plain TRT with a
    Zou-He outlet diverges after ~2,000 steps (oracle and GPU alike).
    """
    t = np.zeros((ny, nx), np.uint8)
    t[:, 0] = INFLOW
    t[:, nx - 1] = OUTFLOW
    t[0, :] = SOLID
    t[ny - 1, :] = SOLID
    cx, cy = nx / 5.0, ny / 2.0
    angle = math.radians(angle_deg)
    _rasterize_ellipse(t, cx, cy, a, b, angle)
    nu = u_in * 2.0 * a / reynolds
    tau = 0.5 + 3.0 * nu
    return Case(q=9, nx=nx, ny=ny, nz=1, types=t.ravel(),
                init=("noise", 1.0, (u_in, 0.0, 0.0), noise, seed, noise_offset), tau=tau, collision=collision, les=les,
                cs_smag=cs_smag, inflow=(u_in, 0.0, 0.0), outflow=1.0, mem=(cx, cy, 0.0, 1.5 * 2.0 * a),
                ref_area=2.0 * a, u_ref=u_in,
                extra={"a": a, "b": b, "angle_deg": angle_deg, "re": reynolds, "ellipse": (cx, cy, a, b, angle)})


def ellipse_sweep_dims(d: int, nx_range=(64, 512), seed: int = BASE_SEED) -> int:
    """NX of the sweep's domain d without building it (ellipse_sweep's first draw)."""
    u0 = float(uniform24(seed + d, 1)[0])
    return int(nx_range[0] + math.floor(u0 * (nx_range[1] - nx_range[0] + 1)))


def ellipse_sweep(n_domains: int = 512, nx_range=(64, 512), seed: int = BASE_SEED, collision: int = 1,
                  first: int = 0, les: bool = True) -> list:
    """The batched sweep: domain d draws from SplitMix64(seed + d) NX ~ U[nx_range] (integer), NY = NX/2,
    semi-axes a in [NY/16, NY/6] and b in [max(NY/16, a/3), a] (aspect a/b in [1, 3]), angle of attack
    ~ U[0, 20] degrees and Re ~ U[50, 300] (outputs 1-5 of the stream), initial noise from output 6 on.
    Domains first .. first + n_domains - 1."""
    cases = []
    for d in range(first, first + n_domains):
        u = uniform24(seed + d, 5).astype(np.float64)
        nx = int(nx_range[0] + math.floor(u[0] * (nx_range[1] - nx_range[0] + 1)))
        ny = nx // 2
        lo, hi = ny / 16.0, ny / 6.0
        a = lo + u[1] * (hi - lo)
        b_lo = max(lo, a / 3.0)
        b = b_lo + u[2] * (a - b_lo)
        angle = 20.0 * u[3]
        re = 50.0 + 250.0 * u[4]
        cases.append(ellipse_channel(nx, ny, a, b, angle, re, collision=collision, les=les, seed=seed + d,
                                     noise_offset=5))
    return cases


def rb_free_fall_velocity(ny: int, rayleigh: float, prandtl: float = 0.71) -> float:
    """Free-fall velocity of a Rayleigh-Benard cell: 0.05, raised (at most to 0.1) until the
    flow's tau - 1/2 = 3 u_ff ny sqrt(Pr / Ra) reaches 0.01, so coarse high-Ra cells stay stable."""
    return min(0.1, max(0.05, 0.01 / (3.0 * ny * math.sqrt(prandtl / rayleigh))))


def rayleigh_benard(nx: int = 128, ny: int = 64, rayleigh: float = 1e4, prandtl: float = 0.71,
                    t_hot: float = 1.0, t_cold: float = 0.0, u_free_fall: float = 0.05, noise: float = 1e-3,
                    collision: int = 1, les: bool = True, cs_smag: float = 0.17, seed: int = BASE_SEED) -> Case:
    """Rayleigh-Benard cell: fluid at rest between a hot wall at y = -1/2 and a cold wall at
    y = ny - 1/2, x periodic, D2Q5 temperature with local Boussinesq buoyancy.

    Parameters as ThermalConvectionScenario (src/scenarios/thermal_convection.cpp:40-48):
    nu * alpha = g beta dT h^3 / Ra, nu = sqrt(nu alpha Pr), alpha = nu / Pr, tau = 3 nu + 1/2,
    with h = ny and g beta = u_ff^2 / (dT h) (free-fall velocity u_ff). The start is the
    conduction profile plus noise * (2 r - 1) from SplitMix64(seed) to trigger convection.
    """
    dT = t_hot - t_cold
    gbeta = u_free_fall ** 2 / (dT * ny)
    nu_alpha = gbeta * dT * ny ** 3 / rayleigh
    nu = math.sqrt(nu_alpha * prandtl)
    alpha = nu / prandtl
    y = (np.arange(ny, dtype=np.float64) + 0.5) / ny
    T = np.repeat(t_hot - dT * y, nx).astype(np.float32)
    T = (T + np.float32(noise) * (np.float32(2.0) * uniform24(seed, nx * ny) - np.float32(1.0))).astype(np.float32)
    t_ref = 0.5 * (t_hot + t_cold)
    return Case(q=9, nx=nx, ny=ny, nz=1, types=np.zeros(nx * ny, np.uint8), init=("uniform", 1.0, (0.0, 0.0, 0.0)),
                tau=0.5 + 3.0 * nu, collision=collision, les=les, cs_smag=cs_smag, u_ref=u_free_fall,
                extra={"thermal": {"tau_t": 0.5 + 3.0 * alpha, "t_ref": t_ref, "beta_g": gbeta, "t_south": t_hot,
                                   "t_north": t_cold}, "T0": T, "ra": rayleigh, "pr": prandtl})


def sphere_channel(nx=256, ny=128, nz=128, radius=12.0, center=(64.0, 64.0, 64.0), u_in=0.05, tau=0.52,
                   collision=1, les=True, cs_smag=0.17, reference_variant=False, device_geometry=False) -> Case:
    """3D sphere in a channel.

    Default: Zou-He inlet u_in on x=0, outlet rho=1 on x=nx-1, periodic y/z,
    TRT + Smagorinsky. ``reference_variant`` gives the form the reference can
    express: x-periodic, y/z half-way walls, no Zou-He, LES not applied.
    ``device_geometry`` leaves the cell types off the host: build_grid types the
    faces and rasterises the sphere on the device (wake_grid_set_solid_sphere),
    which gives the same cells while the sphere stays clear of the faces.
    """
    cx, cy, cz = center
    inflow = outflow = None
    if not reference_variant:
        inflow, outflow = (u_in, 0.0, 0.0), 1.0
    types, extra = None, {}
    if device_geometry and (reference_variant or cx - radius - 1.0 > 0.0 and cx + radius + 1.0 < nx - 1):
        extra["device_sphere"] = (cx, cy, cz, radius)
    else:
        t = np.zeros((nz, ny, nx), np.uint8)
        _rasterize_sphere(t, cx, cy, cz, radius)
        if not reference_variant:
            t[:, :, 0] = np.where(t[:, :, 0] == SOLID, SOLID, INFLOW)
            t[:, :, nx - 1] = np.where(t[:, :, nx - 1] == SOLID, SOLID, OUTFLOW)
        types = t.ravel()
    return Case(q=19, nx=nx, ny=ny, nz=nz, types=types, init=("uniform", 1.0, (u_in, 0.0, 0.0)), tau=tau,
                collision=collision, les=les and not reference_variant, cs_smag=cs_smag, inflow=inflow,
                outflow=outflow, periodic_y=not reference_variant, periodic_z=not reference_variant,
                sphere=(cx, cy, cz, radius), mem=(cx, cy, cz, 2.0 * radius), ref_area=math.pi * radius * radius,
                u_ref=u_in, extra=extra)


def _rasterize_sphere(t: np.ndarray, cx, cy, cz, radius) -> None:
    """LatticeGrid3D::set_solid_sphere (src/grid/lattice_grid_3d.cpp:160-182) in float32."""
    nz, ny, nx = t.shape
    f32 = np.float32
    r_sq = f32(radius) * f32(radius)
    lo = [max(0, int(f32(c) - f32(radius) - f32(1))) for c in (cx, cy, cz)]
    hi = [min(m - 1, int(f32(c) + f32(radius) + f32(1))) for c, m in ((cx, nx), (cy, ny), (cz, nz))]
    zs = np.arange(lo[2], hi[2] + 1)
    ys = np.arange(lo[1], hi[1] + 1)
    xs = np.arange(lo[0], hi[0] + 1)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    dx = X.astype(f32) - f32(cx)
    dy = Y.astype(f32) - f32(cy)
    dz = Z.astype(f32) - f32(cz)
    inside = (dx * dx + dy * dy + dz * dz) <= r_sq
    sub = t[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1]
    sub[inside] = SOLID


def taylor_green(L=384, u0=0.04, tau=0.51, q=27, collision=2) -> Case:
    """Periodic Taylor-Green vortex (form of tests/validation/test_taylor_green_decay.cpp:22-33)."""
    k = 2.0 * math.pi / L
    x = np.arange(L, dtype=np.float64)
    sx, cx_ = np.sin(k * x), np.cos(k * x)
    c2 = np.cos(2 * k * x)
    # broadcast over (z, y, x)
    ux = (u0 * sx[None, None, :] * cx_[None, :, None] * cx_[:, None, None]).astype(np.float32)
    uy = (-u0 * cx_[None, None, :] * sx[None, :, None] * cx_[:, None, None]).astype(np.float32)
    p = (u0 * u0 / 16.0) * (c2[None, None, :] + c2[None, :, None]) * (c2[:, None, None] + 2.0)
    rho = (1.0 + 3.0 * p).astype(np.float32)
    n = L ** 3
    return Case(q=q, nx=L, ny=L, nz=L, types=np.zeros(n, np.uint8),
                init=("fields", rho.ravel(), ux.ravel(), uy.ravel(), np.zeros(n, np.float32)), tau=tau,
                collision=collision, periodic_y=True, periodic_z=True,
                u_ref=u0, extra={"u0": u0, "k": k})


def taylor_green_fields_device(L=384, u0=0.04, device="cuda"):
    """The Taylor-Green fields of ``taylor_green`` computed on the device (FP64, rounded once to
    float32), for lattices too large to build on the host. Returns (rho, ux, uy, uz) CUDA tensors."""
    import torch

    k = 2.0 * math.pi / L
    x = torch.arange(L, dtype=torch.float64, device=device)
    sx, cx_, c2 = torch.sin(k * x), torch.cos(k * x), torch.cos(2 * k * x)
    ux = (u0 * sx[None, None, :] * cx_[None, :, None] * cx_[:, None, None]).float().reshape(-1)
    uy = (-u0 * cx_[None, None, :] * sx[None, :, None] * cx_[:, None, None]).float().reshape(-1)
    p = (u0 * u0 / 16.0) * (c2[None, None, :] + c2[None, :, None]) * (c2[:, None, None] + 2.0)
    rho = (1.0 + 3.0 * p).float().reshape(-1)
    return rho.contiguous(), ux.contiguous(), uy.contiguous(), torch.zeros_like(rho)


def build_grid(case: Case, storage: str = "f32", les_applies: bool = True):
    """Configure a wake_b200 grid for a case (initial state = equilibrium of the fields)."""
    import wake_b200 as wb

    if case.q == 9:
        g = wb.LatticeGrid2D(case.nx, case.ny, case.tau, storage=storage, les_applies=les_applies)
    elif case.q == 19:
        g = wb.LatticeGrid3D(case.nx, case.ny, case.nz, case.tau, storage=storage, les_applies=les_applies)
    else:
        g = wb.LatticeGrid3DQ27(case.nx, case.ny, case.nz, case.tau, storage=storage, les_applies=les_applies)
    kind = case.init[0]
    if kind == "uniform":
        wb.check(wb.lib.wake_grid_initialize(g.handle, case.init[1], *case.init[2]))
    elif kind == "noise":
        _, rho0, u0, amp, seed, off = case.init
        wb.check(wb.lib.wake_grid_initialize_noise(g.handle, rho0, *u0, amp, seed, off))
    else:
        g.initialize_fields(case.rho, case.ux, case.uy, case.uz if case.q != 9 else None)
    host_types = case.types is not None
    if host_types:
        g.set_cell_types(case.types)
    if case.q != 9 and (case.periodic_y or case.periodic_z):
        g.set_periodic_axes(case.periodic_y, case.periodic_z)
    if case.inflow is not None:
        wb.check(wb.lib.wake_grid_set_inflow_west(g.handle, *case.inflow))
        if host_types:
            g.set_cell_types(case.types)  # keep the case's exact typing of the faces
    if case.outflow is not None:
        g.set_outflow_east(case.outflow)
        if host_types:
            g.set_cell_types(case.types)
    if case.extra.get("device_sphere") is not None:
        g.set_solid_sphere(*case.extra["device_sphere"])
    if case.sphere is not None and case.q == 19:
        g.build_curved_sphere_links(*case.sphere)
    if case.mem is not None:
        g.enable_forces(*case.mem)
    th = case.extra.get("thermal")
    if th is not None:
        g.enable_thermal(th["tau_t"], th["t_ref"], th["beta_g"], th["t_south"], th["t_north"])
        if case.extra.get("T0") is not None:
            g.initialize_temperature(case.extra["T0"])
    return g
