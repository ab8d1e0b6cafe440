"""Host-side logic of the batched / served workloads (no GPU needed)."""
import math

import numpy as np

from wake_b200 import serve as S
from wake_b200 import workloads as W


def test_mixed_jobs_are_deterministic_and_lazy():
    a = S.mixed_jobs(50, 20.0)
    b = S.mixed_jobs(50, 20.0)
    assert [(j.kind, j.dims, j.steps, j.arrival) for j in a] == [(j.kind, j.dims, j.steps, j.arrival) for j in b]
    assert all(a[i].arrival < a[i + 1].arrival for i in range(49))
    c = a[0].make()
    assert (c.q, c.nx, c.ny, c.nz) == a[0].dims


def test_mixed_jobs_distribution():
    jobs = S.mixed_jobs(2000, 100.0)
    steps = np.array([j.steps for j in jobs])
    assert steps.min() >= 200 and steps.max() <= 20000
    assert abs(np.median(steps) / 2000.0 - 1.0) < 0.1
    assert abs(np.percentile(steps, 5) / 500.0 - 1.0) < 0.15
    frac3d = np.mean([j.kind == "d3q19" for j in jobs])
    assert abs(frac3d - 0.5) < 0.05
    n2 = [j for j in jobs if j.kind != "d3q19"]
    assert abs(np.mean([j.kind == "thermal" for j in n2]) - 0.1) < 0.03
    n3 = np.array([j.dims[1] for j in jobs if j.kind == "d3q19"])
    assert n3.min() >= 48 and n3.max() <= 160 and all(j.dims[1] == j.dims[2] == j.dims[3] for j in jobs
                                                       if j.kind == "d3q19")
    nx2 = np.array([j.dims[1] for j in jobs if j.kind != "d3q19"])
    assert nx2.min() >= 64 and nx2.max() <= 512
    assert all(j.dims[2] == j.dims[1] // 2 for j in jobs if j.kind != "d3q19")
    gaps = np.diff([0.0] + [j.arrival for j in jobs])
    assert abs(gaps.mean() * 100.0 - 1.0) < 0.1  # Poisson process at 100 jobs/s


def test_sweep_dims_match_built_domains():
    for d in range(20):
        c = W.ellipse_sweep(1, first=d)[0]
        assert c.nx == W.ellipse_sweep_dims(d) and c.ny == c.nx // 2
        a, b = c.extra["a"], c.extra["b"]
        assert c.ny / 16 - 1e-9 <= b <= a <= c.ny / 6 + 1e-9 and a / b <= 3.0 + 1e-9
        assert 0.0 <= c.extra["angle_deg"] <= 20.0 and 50.0 <= c.extra["re"] <= 300.0
        assert math.isclose(c.tau, 0.5 + 3.0 * 0.05 * 2.0 * a / c.extra["re"])


def test_memory_estimate_covers_state_buffers():
    for q, dims in ((9, (300, 150, 1)), (19, (64, 64, 64)), (27, (32, 32, 32))):
        n = dims[0] * dims[1] * dims[2]
        for storage, elem in ((0, 4), (1, 2), (2, 2)):
            est = S.lib.wake_grid_estimate_bytes(q, *dims, storage, 0)
            assert est >= 2 * q * n * elem + q * n * 4
            assert S.lib.wake_grid_estimate_bytes(q, *dims, storage, 1) == est + 20 * n
    assert S.lib.wake_grid_estimate_bytes(10, 8, 8, 8, 0, 0) < 0
    S.lib.wake_gpu_clear_error()


def test_thermal_jobs_build_rayleigh_benard_cells():
    jobs = [j for j in S.mixed_jobs(400, 50.0) if j.kind == "thermal"]
    assert jobs
    for j in jobs[:5]:
        c = j.make()
        assert (c.nx, c.ny) == (j.dims[1], j.dims[2]) and "thermal" in c.extra
        assert 1e4 <= c.extra["ra"] <= 1e6 and c.tau - 0.5 >= 0.0079 and c.extra["thermal"]["tau_t"] > 0.5
        assert S.job_bytes(j, "f32") > S.lib.wake_grid_estimate_bytes(9, c.nx, c.ny, 1, 0, 0)
