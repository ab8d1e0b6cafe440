"""Python mirror of the reference's lattice classes over the fused GPU engine.

``LatticeGrid2D`` / ``LatticeGrid3D`` keep the method names, argument order and
defaults of wake::LatticeGrid2D (include/wake/grid/lattice_grid_2d.hpp:14-113)
and wake::LatticeGrid3D (include/wake/grid/lattice_grid_3d.hpp:20-123). The
state lives on the GPU; field accessors copy the reference-visible arrays
(f_src, rho, u, speed after the last step) back as numpy arrays.

One behavioural choice differs from the reference and is explicit: the
reference computes the Smagorinsky tau when ``use_les`` is true but never
passes it to the collision (src/grid/lattice_grid_2d.cpp:205-210). Here
``les_applies=True`` (default) applies it per node; ``les_applies=False``
reproduces the reference, where ``use_les`` changes nothing.
"""
from __future__ import annotations

import numpy as np

from ._lib import addr, check, lib

BGK, TRT, MRT = 0, 1, 2
FLUID, SOLID, INFLOW, OUTFLOW, MOVING_WALL = 0, 1, 2, 3, 6
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f16c": 3}
DEFAULT_SMAGORINSKY_CONSTANT = 0.14  # include/wake/core/constants.hpp:22


class _Grid:
    Q = 0

    def __init__(self, nx: int, ny: int, nz: int, relaxation_time: float, storage: str, les_applies: bool):
        self._h = lib.wake_grid_create(self.Q, nx, ny, nz, float(relaxation_time), STORAGE[storage])
        if not self._h:
            check(-1)
        self.nx, self.ny, self.nz = nx, ny, nz
        self._tau = float(relaxation_time)
        self.storage = storage
        self.les_applies = les_applies
        self._model = None
        self._tau_bulk = 1.63 if self.Q == 9 else (1.19 if self.Q == 19 else 1.0)
        self.lambda_trt = 0.25
        self.mrt_exact = False
        self.s3 = 1.0
        self.s4 = 1.0

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            batch = getattr(self, "_batch", None)
            if batch is not None and batch.handle:
                batch.remove(self)  # a member must leave its batch before it is destroyed
            lib.wake_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- sizes and parameters
    def total_nodes(self) -> int:
        return self.nx * self.ny * self.nz

    def current_step(self) -> int:
        return int(lib.wake_grid_step_count(self._h))

    def relaxation_time(self) -> float:
        return self._tau

    def set_relaxation_time(self, tau: float) -> None:
        self._tau = float(tau)
        check(lib.wake_grid_set_relaxation_time(self._h, self._tau))

    def kinematic_viscosity(self) -> float:
        return (1.0 / 3.0) * (self._tau - 0.5)

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.wake_grid_set_stream(self._h, stream_ptr))

    def set_tau_bulk(self, tau_bulk: float) -> None:
        self._tau_bulk = float(tau_bulk)
        self._model = None

    # -- initialisation
    def initialize(self, rho_init=1.0, ux_init=0.0, uy_init=0.0, uz_init=0.0) -> None:
        check(lib.wake_grid_initialize(self._h, rho_init, ux_init, uy_init, uz_init))

    def initialize_fields(self, rho, ux, uy, uz=None) -> None:
        """Initial populations = equilibrium of the fields (numpy arrays, or contiguous float32 CUDA tensors)."""
        def prep(a):
            if a is None or (hasattr(a, "data_ptr") and getattr(a, "is_cuda", False)):
                if a is not None and (a.dtype.itemsize != 4 or not a.is_contiguous() or a.numel() != self.total_nodes()):
                    raise ValueError("device fields must be contiguous float32 tensors of one value per node")
                return a
            return np.ascontiguousarray(a, dtype=np.float32).ravel()

        arrs = [prep(a) for a in (rho, ux, uy, uz)]
        check(lib.wake_grid_initialize_fields(self._h, *[addr(a) for a in arrs]))

    def set_populations(self, f) -> None:
        """Set the reference-visible populations f_src, layout [q][node]."""
        if hasattr(f, "data_ptr") and getattr(f, "is_cuda", False):
            check(lib.wake_grid_set_populations_device(self._h, f.data_ptr()))
            return
        f = np.ascontiguousarray(f, dtype=np.float32)
        check(lib.wake_grid_set_populations(self._h, addr(f)))

    # -- geometry
    def set_cell_types(self, types) -> None:
        t = np.ascontiguousarray(types, dtype=np.uint8).ravel()
        check(lib.wake_grid_set_cell_types(self._h, addr(t)))

    def cell_type_data(self) -> np.ndarray:
        t = np.empty(self.total_nodes(), dtype=np.uint8)
        check(lib.wake_grid_get_cell_types(self._h, addr(t)))
        return t

    def set_outflow_east(self, rho_out=1.0) -> None:
        check(lib.wake_grid_set_outflow_east(self._h, rho_out))

    # -- forces
    def enable_forces(self, cx, cy, cz=0.0, r_max=0.0, capacity=1 << 16) -> None:
        check(lib.wake_grid_enable_forces(self._h, cx, cy, cz, r_max, capacity))

    def force_history(self) -> np.ndarray:
        n = int(lib.wake_grid_force_count(self._h))
        out = np.zeros((max(n, 1), 3), dtype=np.float64)
        got = check(lib.wake_grid_get_force_history(self._h, addr(out), out.shape[0]))
        return out[:got]

    # -- stepping
    def _apply_model(self, collision: int, use_les: bool, smag_const: float) -> None:
        model = (collision, bool(use_les and self.les_applies), float(smag_const), self._tau_bulk, self.lambda_trt,
                 self.mrt_exact, self.s3, self.s4)
        if model != self._model:
            check(lib.wake_grid_set_model(self._h, collision, int(model[1]), smag_const, self.lambda_trt,
                                          self._tau_bulk, int(self.mrt_exact), self.s3, self.s4))
            self._model = model

    def use_graph(self, steps_per_graph: int) -> None:
        check(lib.wake_grid_use_graph(self._h, steps_per_graph))

    def prepare_steps(self, collision=MRT, gx=0.0, gy=0.0, gz=0.0, use_les=False,
                      smag_const=DEFAULT_SMAGORINSKY_CONSTANT) -> None:
        """Do the one-time work of the next step() with these arguments now (re-collision after a
        change, graph capture); advances nothing (wake_grid_prepare_steps)."""
        self._apply_model(collision, use_les, smag_const)
        check(lib.wake_grid_prepare_steps(self._h, gx, gy, gz))

    def synchronize(self) -> None:
        check(lib.wake_grid_synchronize(self._h))

    # -- reference-visible state
    def f_src_data(self) -> np.ndarray:
        f = np.empty((self.Q, self.total_nodes()), dtype=np.float32)
        check(lib.wake_grid_get_populations(self._h, addr(f)))
        return f

    def macroscopic(self) -> dict:
        n = self.total_nodes()
        out = {k: np.empty(n, dtype=np.float32) for k in ("rho", "ux", "uy", "uz", "speed")}
        check(lib.wake_grid_get_macroscopic(self._h, addr(out["rho"]), addr(out["ux"]), addr(out["uy"]),
                                            addr(out["uz"]) if self.Q != 9 else None, addr(out["speed"])))
        if self.Q == 9:
            del out["uz"]
        return out

    macro = macroscopic

    def macroscopic_into(self, rho=None, ux=None, uy=None, uz=None, speed=None) -> None:
        """Copy the moments after the last step into caller buffers (host arrays or CUDA tensors of one
        float32 per node); a None buffer is skipped."""
        for a in (rho, ux, uy, uz, speed):
            if a is not None and (a.dtype.itemsize != 4 or (a.numel() if hasattr(a, "numel") else a.size)
                                  != self.total_nodes()):
                raise ValueError("moment buffers hold one float32 per node")
        check(lib.wake_grid_get_macroscopic(self._h, addr(rho), addr(ux), addr(uy),
                                            addr(uz) if self.Q != 9 else None, addr(speed)))

    def rho_data(self) -> np.ndarray:
        return self.macroscopic()["rho"]

    def ux_data(self) -> np.ndarray:
        return self.macroscopic()["ux"]

    def uy_data(self) -> np.ndarray:
        return self.macroscopic()["uy"]

    def speed_data(self) -> np.ndarray:
        return self.macroscopic()["speed"]

    def _diag(self):
        import ctypes as C

        m, ke, mx = C.c_double(), C.c_double(), C.c_double()
        check(lib.wake_grid_diagnostics(self._h, C.addressof(m), C.addressof(ke), C.addressof(mx)))
        return m.value, ke.value, mx.value

    def compute_total_mass(self) -> float:
        return self._diag()[0]

    def compute_total_kinetic_energy(self) -> float:
        return self._diag()[1]

    def compute_max_speed(self) -> float:
        return self._diag()[2]

    def total_mass_all(self) -> float:
        import ctypes as C

        m = C.c_double()
        check(lib.wake_grid_total_mass(self._h, C.addressof(m)))
        return m.value


class LatticeGrid2D(_Grid):
    """GPU counterpart of wake::LatticeGrid2D (src/grid/lattice_grid_2d.cpp:46-295)."""

    Q = 9

    def __init__(self, nx: int, ny: int, relaxation_time: float = 0.6, storage: str = "f32", les_applies: bool = True):
        super().__init__(nx, ny, 1, relaxation_time, storage, les_applies)

    def step(self, collision=MRT, gx=0.0, gy=0.0, use_les=False, smag_const=DEFAULT_SMAGORINSKY_CONSTANT, n=1):
        self._apply_model(collision, use_les, smag_const)
        check(lib.wake_grid_step(self._h, n, gx, gy, 0.0))

    def update_macroscopic(self) -> None:
        """Nothing to do: every accessor reads the state of the last step."""

    def initialize_custom(self, init_fn) -> None:
        rho = np.empty((self.ny, self.nx), np.float32)
        ux = np.empty_like(rho)
        uy = np.empty_like(rho)
        for y in range(self.ny):
            for x in range(self.nx):
                rho[y, x], ux[y, x], uy[y, x] = init_fn(x, y)
        self.initialize_fields(rho, ux, uy)

    def set_cell_type(self, x: int, y: int, t: int) -> None:
        check(lib.wake_grid_set_cell_type(self._h, x, y, 0, t))

    def get_cell_type(self, x: int, y: int) -> int:
        if 0 <= x < self.nx and 0 <= y < self.ny:
            return int(self.cell_type_data()[y * self.nx + x])
        return SOLID

    def set_solid_box(self, x0, y0, x1, y1) -> None:
        check(lib.wake_grid_set_solid_box(self._h, x0, y0, 0, x1, y1, 0))

    def set_solid_circle(self, cx, cy, radius) -> None:
        check(lib.wake_grid_set_solid_circle(self._h, cx, cy, radius))

    def set_inflow_west(self, u_in_x, u_in_y=0.0) -> None:
        check(lib.wake_grid_set_inflow_west(self._h, u_in_x, u_in_y, 0.0))

    def set_moving_wall_north(self, u_wall_x) -> None:
        check(lib.wake_grid_set_moving_wall(self._h, u_wall_x, 0.0, 0.0))

    # -- coupled temperature (D2Q5 with local Boussinesq force; see wake_grid_enable_thermal)
    def enable_thermal(self, tau_thermal: float, t_ref: float = 0.5, beta_g: float = 0.0,
                       t_hot_south: float = 1.0, t_cold_north: float = 0.0) -> None:
        """Couple a temperature field to the flow: buoyancy beta_g (T - t_ref) along +y per node,
        isothermal walls y = -1/2 (t_hot_south) and y = ny - 1/2 (t_cold_north). Before the first step."""
        check(lib.wake_grid_enable_thermal(self._h, tau_thermal, t_ref, beta_g, t_hot_south, t_cold_north))
        self._thermal = (float(t_hot_south), float(t_cold_north))

    def initialize_temperature(self, T) -> None:
        arr = np.ascontiguousarray(T, dtype=np.float32).ravel()
        check(lib.wake_grid_initialize_temperature(self._h, addr(arr)))

    def temperature_data(self) -> np.ndarray:
        out = np.empty(self.total_nodes(), np.float32)
        check(lib.wake_grid_get_temperature(self._h, addr(out)))
        return out

    def compute_nusselt_number(self) -> float:
        """Hot-wall Nusselt number: mean temperature drop between the first two rows over the
        conduction drop (the form of ThermalSolver2D::compute_nusselt_number,
        src/thermal/thermal_solver.cpp:131-146). The walls here sit half a cell outside the
        first and last rows, so conduction drops (t_hot - t_cold) / ny per row, where the
        reference, whose walls are the first and last rows, divides by ny - 1."""
        t_hot, t_cold = getattr(self, "_thermal", (1.0, 0.0))
        if abs(t_hot - t_cold) < 1e-6 or self.ny <= 1:
            return 1.0
        T = self.temperature_data().reshape(self.ny, self.nx).astype(np.float64)
        mean_grad = float(np.mean(T[0] - T[1]))
        return mean_grad / ((t_hot - t_cold) / self.ny)


class LatticeGrid3D(_Grid):
    """GPU counterpart of wake::LatticeGrid3D (src/grid/lattice_grid_3d.cpp:46-410).

    Beyond the reference: ``set_periodic_axes`` wraps y / z with solids present
    and ``set_inflow_west`` / ``set_outflow_east`` apply D3Q19 Zou-He faces.
    """

    Q = 19

    def __init__(self, nx, ny, nz, relaxation_time=0.6, storage="f32", les_applies=True):
        super().__init__(nx, ny, nz, relaxation_time, storage, les_applies)
        self._periodic = True

    def step(self, collision=MRT, gx=0.0, gy=0.0, gz=0.0, use_les=False, smag_const=DEFAULT_SMAGORINSKY_CONSTANT,
             n=1):
        self._apply_model(collision, use_les, smag_const)
        check(lib.wake_grid_step(self._h, n, gx, gy, gz))

    def update_macroscopic(self) -> None:
        """Nothing to do: every accessor reads the state of the last step."""

    def set_periodic_axes(self, periodic_y: bool, periodic_z: bool) -> None:
        check(lib.wake_grid_set_periodic(self._h, int(periodic_y), int(periodic_z)))

    def set_cell_type(self, x, y, z, t) -> None:
        check(lib.wake_grid_set_cell_type(self._h, x, y, z, t))

    def set_solid_box(self, x0, y0, z0, x1, y1, z1) -> None:
        check(lib.wake_grid_set_solid_box(self._h, x0, y0, z0, x1, y1, z1))

    def set_solid_sphere(self, cx, cy, cz, radius) -> None:
        check(lib.wake_grid_set_solid_sphere(self._h, cx, cy, cz, radius))

    def set_moving_wall_top(self, u_wall_x, u_wall_z=0.0) -> None:
        check(lib.wake_grid_set_moving_wall(self._h, u_wall_x, 0.0, u_wall_z))

    def set_inflow_west(self, ux, uy=0.0, uz=0.0) -> None:
        check(lib.wake_grid_set_inflow_west(self._h, ux, uy, uz))

    def build_curved_sphere_links(self, cx, cy, cz, radius) -> int:
        check(lib.wake_grid_build_curved_sphere_links(self._h, cx, cy, cz, radius))
        return int(lib.wake_grid_num_curved_links(self._h))

    def set_curved_links(self, idx, q, delta, uw=None) -> None:
        idx = np.ascontiguousarray(idx, np.int32)
        q = np.ascontiguousarray(q, np.int32)
        delta = np.ascontiguousarray(delta, np.float32)
        u = [None, None, None]
        if uw is not None:
            uw = np.asarray(uw, np.float32)
            u = [np.ascontiguousarray(uw[:, a]) for a in range(3)]
        check(lib.wake_grid_set_curved_links(self._h, len(idx), addr(idx), addr(q), addr(delta), *[addr(a) for a in u]))

    def curved_links(self):
        n = int(lib.wake_grid_num_curved_links(self._h))
        idx = np.empty(n, np.int32)
        q = np.empty(n, np.int32)
        d = np.empty(n, np.float32)
        lib.wake_grid_get_curved_links(self._h, addr(idx), addr(q), addr(d))
        return idx, q, d

    def uz_data(self) -> np.ndarray:
        return self.macroscopic()["uz"]


class LatticeGrid3DQ27(LatticeGrid3D):
    """D3Q27 lattice on the same engine (the reference has D3Q27 kernels but no grid)."""

    Q = 27
