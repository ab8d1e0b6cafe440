"""Allocation-free momentum exchange, checked against the allocating entry point.

d3q19_compute_momentum_exchange_forces_noalloc serves callers that cannot
allocate device memory while they run (a serving loop that has committed all of
HBM to resident lattices, or a latency-critical loop where cudaMalloc would
synchronise the device). It keeps its partial sums in a fixed array of the
library instead. These tests call it through the C ABI with device buffers and
compare it with d3q19_compute_momentum_exchange_forces on the same inputs, on
two calls in a row with different inputs (the shared array keeps the previous
call's contents, which must not leak into the next result), with the
reference's own output on the per-call fixture, and at its node limit.

The file name sorts last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

wb = pytest.importorskip("wake_b200")
torch = pytest.importorskip("torch")
from wake_b200 import workloads as W  # noqa: E402

WEIGHTS = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)


def _noalloc():
    fn = wb.lib.d3q19_compute_momentum_exchange_forces_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def _inputs(seed, nx, ny, nz, center, radius):
    n = nx * ny * nz
    noise = W.uniform24(seed, 19 * n).reshape(19, n)
    f = (WEIGHTS[:, None] * (1.0 + 0.2 * (noise - 0.5))).astype(np.float32)
    t = np.zeros((nz, ny, nx), np.uint8)
    W._rasterize_sphere(t, *center, radius)
    return torch.from_numpy(f).cuda(), torch.from_numpy(t.ravel()).cuda()


def _both(fn, f, ct, nx, ny, nz, center, r_max):
    """(no-alloc result, allocating entry point's result) on the same device buffers."""
    ref = [torch.zeros(1, device="cuda") for _ in range(3)]
    wb.lib.d3q19_compute_momentum_exchange_forces(f.data_ptr(), ct.data_ptr(), nx, ny, nz, *center, r_max,
                                                  *[r.data_ptr() for r in ref])
    out = [torch.full((1,), float("nan"), device="cuda") for _ in range(3)]
    rc = fn(f.data_ptr(), ct.data_ptr(), nx, ny, nz, *center, r_max, *[o.data_ptr() for o in out])
    assert rc == 0, wb.lib.wake_gpu_last_error()
    return np.array([o.item() for o in out]), np.array([r.item() for r in ref])


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    """A larger lattice first (1152 partial sums), then a smaller one (144): the second result
    must not see the first call's partials. Up to 303,104 nodes both entry points add the same
    partials in the same order, so the results are equal bit for bit."""
    fn = _noalloc()
    for (nx, ny, nz), center, radius, r_max, seed in (((96, 64, 48), (40.0, 32.0, 24.0), 10.0, 20.0, 11),
                                                      ((48, 32, 24), (20.0, 16.0, 12.0), 6.0, 12.0, 12)):
        f, ct = _inputs(W.BASE_SEED + seed, nx, ny, nz, center, radius)
        got, exp = _both(fn, f, ct, nx, ny, nz, center, r_max)
        assert np.all(np.isfinite(got)) and np.any(got != 0.0)
        assert np.array_equal(got, exp), (got, exp)


def test_noalloc_matches_reference_output(golden):
    """The reference's own momentum exchange on the per-call fixture (10 x 8 x 6 lattice)."""
    d = golden("percall")
    fn = _noalloc()
    f = torch.from_numpy(d["s3_f"]).cuda()
    ct = torch.from_numpy(d["s3_ct"]).cuda()
    out = [torch.zeros(1, device="cuda") for _ in range(3)]
    rc = fn(f.data_ptr(), ct.data_ptr(), 10, 8, 6, 4.5, 3.5, 2.5, 0.0, *[o.data_ptr() for o in out])
    assert rc == 0, wb.lib.wake_gpu_last_error()
    got = np.array([o.item() for o in out])
    # same bound as the allocating entry point's parity test against this fixture
    assert np.allclose(got, d["s3_mem"], rtol=1e-5, atol=1e-6), (got, d["s3_mem"])


def test_noalloc_at_its_node_limit():
    """Exactly 4,194,304 nodes (the 256 x 128 x 128 sphere channel), the largest size accepted.
    The allocating entry point adds 1184 partial sums where this one adds 16384, so the two
    agree to FP64 rounding of the sums, far inside the parity bound used against the reference."""
    fn = _noalloc()
    nx, ny, nz = 256, 128, 128
    center = (64.0, 64.0, 64.0)
    f, ct = _inputs(W.BASE_SEED + 14, nx, ny, nz, center, 12.0)
    got, exp = _both(fn, f, ct, nx, ny, nz, center, 24.0)
    assert np.all(np.isfinite(got)) and np.any(got != 0.0)
    assert np.allclose(got, exp, rtol=1e-6, atol=1e-7), (got, exp)
    del f, ct
    torch.cuda.empty_cache()


def test_noalloc_rejects_what_it_cannot_serve():
    fn = _noalloc()
    f, ct = _inputs(W.BASE_SEED + 13, 8, 8, 8, (4.0, 4.0, 4.0), 2.0)
    out = [torch.zeros(1, device="cuda") for _ in range(3)]
    # more nodes than the fixed scratch holds: refused before any device access
    wb.lib.wake_gpu_clear_error()
    rc = fn(f.data_ptr(), ct.data_ptr(), 256, 128, 129, 4.0, 4.0, 4.0, 0.0, *[o.data_ptr() for o in out])
    assert rc == -1 and b"scratch limit" in wb.lib.wake_gpu_last_error()
    # host memory would need staging, which allocates: refused
    host = np.zeros(3, np.float32)
    rc = fn(f.data_ptr(), ct.data_ptr(), 8, 8, 8, 4.0, 4.0, 4.0, 0.0, host.ctypes.data, host.ctypes.data + 4,
            host.ctypes.data + 8)
    assert rc == -1
    wb.lib.wake_gpu_clear_error()
