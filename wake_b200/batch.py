"""Many resident lattices advanced together (C ABI ``wake_batch_*``).

A ``Batch`` holds grids of one lattice and storage (``LatticeGrid2D`` /
``LatticeGrid3D`` / ``LatticeGrid3DQ27`` objects) and advances all of them with
one bulk launch, one general launch and one force reduction per step,
whatever their sizes. Each member keeps its own geometry, tau, boundaries and
force history and is read through its usual accessors between steps; its
results are the ones it gets when stepped alone.

There is no reference counterpart: the reference runs one LatticeGrid per
object and step call (src/grid/lattice_grid_2d.cpp:195-265,
src/runner/runner.cpp:136).
"""
from __future__ import annotations

import ctypes

from ._lib import check, lib
from .grid import DEFAULT_SMAGORINSKY_CONSTANT, STORAGE, TRT


class Batch:
    def __init__(self, q: int = 9, storage: str = "f32"):
        self._h = lib.wake_batch_create(q, STORAGE[storage])
        if not self._h:
            check(-1)
        self.q = q
        self.storage = storage
        self._members: list = []

    # -- lifetime
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.wake_batch_destroy(self._h)
            self._h = None
            for g in self._members:
                g._batch = None
            self._members = []

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- membership
    def add(self, grid, collision: int = TRT, use_les: bool = False,
            smag_const: float = DEFAULT_SMAGORINSKY_CONSTANT) -> int:
        """Add a grid; its collision model is set like grid.step(collision, use_les=...) would."""
        grid._apply_model(collision, use_les, smag_const)
        idx = check(lib.wake_batch_add(self._h, grid.handle))
        self._members.append(grid)
        grid._batch = self
        return idx

    def remove(self, grid) -> None:
        check(lib.wake_batch_remove(self._h, grid.handle))
        self._members = [g for g in self._members if g is not grid]
        grid._batch = None

    def __len__(self) -> int:
        return len(self._members)

    @property
    def members(self) -> list:
        return list(self._members)

    # -- stepping
    def step(self, n: int = 1) -> None:
        check(lib.wake_batch_step(self._h, n))

    def use_graph(self, steps_per_graph: int) -> None:
        check(lib.wake_batch_use_graph(self._h, steps_per_graph))

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib.wake_batch_set_stream(self._h, stream_ptr))

    def set_block(self, threads_bulk: int, threads_general: int = 128) -> None:
        check(lib.wake_batch_set_block(self._h, threads_bulk, threads_general))

    def block(self) -> int:
        return check(lib.wake_batch_get_block(self._h))

    def autotune(self, steps: int = 20) -> int:
        """Pick the bulk block size by timing real steps (members advance `steps` per size tried)."""
        best = ctypes.c_int()
        check(lib.wake_batch_autotune(self._h, steps, ctypes.byref(best)))
        return best.value

    def host_seconds(self) -> dict:
        """Host time spent inside step() so far: member/table preparation, graph capture, launches."""
        v = [ctypes.c_double() for _ in range(3)]
        check(lib.wake_batch_host_seconds(self._h, *[ctypes.byref(x) for x in v]))
        return {"prepare": v[0].value, "capture": v[1].value, "launch": v[2].value}

    def synchronize(self) -> None:
        check(lib.wake_batch_synchronize(self._h))

    def info(self) -> dict:
        nodes, fr, gr, lps = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib.wake_batch_info(self._h, ctypes.byref(nodes), ctypes.byref(fr), ctypes.byref(gr), ctypes.byref(lps)))
        return {"members": len(self._members), "nodes": nodes.value, "bulk_rows": fr.value, "general_rows": gr.value,
                "launches_per_step": lps.value}
