"""Continuous-batching server: every job's result is the same in the mix as alone.

Jobs of two kinds (D2Q9 channels, D3Q19 sphere channels) with different sizes
and step counts go through the server under an HBM budget that holds only part
of them at once, so admission waits for departures and batches change
membership every few ticks. Each job's per-step force history and FP64
diagnostics must equal, bit for bit, those of the job run alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

wb = pytest.importorskip("wake_b200")
from wake_b200 import serve as S  # noqa: E402


def _small_mix(n=10, rate=200.0, thermal_frac=0.1):
    return S.mixed_jobs(n, rate, n_range=(16, 28), nx_range=(64, 128), median_steps=60.0, p5_steps=20.0,
                        steps_range=(10, 200), thermal_frac=thermal_frac)


def _assert_same(a, b):
    assert a.error is None and b.error is None, (a.error, b.error)
    if a.kind == "thermal":  # no obstacle, no force monitor; the wall heat flux instead
        assert a.nusselt is not None and a.nusselt == b.nusselt, f"job {a.id}: Nusselt number differs"
    else:
        assert a.forces.shape == (a.steps, 3)
    assert np.array_equal(a.forces, b.forces), f"job {a.id}: force history differs"
    assert a.diagnostics == b.diagnostics, f"job {a.id}: diagnostics differ"


def test_results_identical_alone_and_in_the_mix():
    jobs = _small_mix(12, thermal_frac=0.4)
    assert "thermal" in {j.kind for j in jobs}
    assert {"d2q9", "d3q19"} <= {j.kind for j in jobs}
    need = [S.job_bytes(j, "f32") for j in jobs]
    budget = int(0.5 * sum(need))  # about half the jobs resident at once
    assert budget >= max(need)
    rep = S.Server(budget, max_tick_steps=16).run(jobs, realtime=False)
    assert len(rep.results) == len(jobs)
    assert rep.peak_resident_bytes <= budget
    alone = {j.id: S.run_alone(j) for j in jobs}
    for r in rep.results:
        _assert_same(r, alone[r.id])


def test_realtime_poisson_arrivals_complete_with_latencies():
    jobs = _small_mix(12, rate=400.0)
    budget = sum(S.job_bytes(j, "f32") for j in jobs)
    rep = S.Server(budget, max_tick_steps=32).run(jobs, realtime=True)
    s = rep.summary()
    assert s["jobs"] == 12 and s["failed"] == 0, [(r.id, r.kind, r.error) for r in rep.results if r.error]
    assert all(r.completed >= r.admitted >= r.arrival - 1e-9 for r in rep.results)
    assert 0.0 < s["p50_latency_s"] <= s["p99_latency_s"]


def test_job_larger_than_budget_is_refused_and_others_run():
    jobs = _small_mix(4)
    small = min(S.job_bytes(j, "f32") for j in jobs)
    rep = S.Server(small, max_tick_steps=16).run(jobs, realtime=False)
    errs = [r for r in rep.results if r.error]
    ok = [r for r in rep.results if r.error is None]
    assert ok and all("budget" in r.error for r in errs)


def test_fp16_mix_matches_fp16_alone():
    jobs = _small_mix(6)
    rep = S.Server(sum(S.job_bytes(j, "f16") for j in jobs), storage="f16", max_tick_steps=8).run(jobs,
                                                                                                    realtime=False)
    for r in rep.results:
        _assert_same(r, S.run_alone(next(j for j in jobs if j.id == r.id), storage="f16"))
