"""Continuous-batching simulation server over resident lattices.

Jobs (a lattice case plus a step count) arrive over time. The server admits
them in arrival order while their device memory fits a fixed HBM budget and a
slot is free, keeps each admitted lattice resident, and advances all resident
jobs of one kind (lattice, collision model, LES switch) together as one
``Batch``: a tick steps every batch by the smallest number of steps any of its
members still needs (capped), so each job runs exactly its step count and
leaves as soon as it is done, freeing memory for the next arrivals. Batches of
different kinds run concurrently on their own streams.

Results of a job (its per-step force history and FP64 diagnostics) are the
same bits it gets when run alone: members of a batch run the single-lattice
arithmetic (wake_batch_* in include/wake_gpu.h).

The reference has no server: it runs one scenario per process
(src/runner/runner.cpp:136-183).
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from ._lib import check, lib
from .batch import Batch
from .grid import STORAGE


@dataclass
class Job:
    """A simulation request. The lattice case is built on admission (``make()``), so a
    long arrival list costs no host memory until its jobs are admitted."""

    id: int
    kind: str            # "d2q9" | "thermal" | "d3q19"
    dims: tuple          # (q, nx, ny, nz)
    make: object         # () -> workloads.Case
    steps: int
    arrival: float = 0.0  # seconds after the start of the run
    model: tuple = (1, True, 0.17)  # (collision, LES, Cs): jobs of one model share a batch

    @property
    def nodes(self) -> int:
        return self.dims[1] * self.dims[2] * self.dims[3]


def job_from_case(jid: int, kind: str, case: W.Case, steps: int, arrival: float = 0.0) -> Job:
    return Job(jid, kind, (case.q, case.nx, case.ny, case.nz), lambda: case, steps, arrival,
               (case.collision, bool(case.les), case.cs_smag))


@dataclass
class JobResult:
    id: int
    kind: str
    steps: int
    arrival: float
    admitted: float
    completed: float
    forces: np.ndarray           # [steps, 3] FP64 (Fx, Fy, Tz) or (Fx, Fy, Fz)
    diagnostics: tuple           # (mass, kinetic energy, max speed) in FP64 over fluid nodes
    error: str | None = None
    nodes: int = 0
    nusselt: float | None = None  # Rayleigh-Benard jobs: hot-wall Nusselt number at the end

    @property
    def latency(self) -> float:
        return self.completed - self.arrival


@dataclass
class ServeReport:
    results: list
    makespan: float
    ticks: int
    peak_resident_bytes: int
    budget_bytes: int
    extra: dict = field(default_factory=dict)

    def summary(self) -> dict:
        lat = np.array([r.latency for r in self.results]) if self.results else np.zeros(1)
        done = [r for r in self.results if r.error is None]
        failed = [[r.id, r.kind, (r.error or "")[:160]] for r in self.results if r.error is not None]
        return {"jobs": len(self.results), "failed": len(failed), "failed_jobs": failed[:10],
                "sims_per_s": len(self.results) / self.makespan if self.makespan > 0 else 0.0,
                "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                "mean_latency_s": float(lat.mean()), "makespan_s": self.makespan, "ticks": self.ticks,
                "peak_resident_bytes": self.peak_resident_bytes, "budget_bytes": self.budget_bytes,
                "node_steps": int(sum(r.steps * r.nodes for r in done)), **self.extra}


# ------------------------------------------------------------------ workload
def lognormal_steps(u1: float, u2: float, median: float = 2000.0, p5: float = 500.0, lo: int = 200,
                    hi: int = 20000) -> int:
    """Steps ~ lognormal(median, sigma with 5th percentile p5), clipped to [lo, hi] (Box-Muller on two uniforms)."""
    sigma = math.log(median / p5) / 1.6448536269514722
    z = math.sqrt(-2.0 * math.log(max(u1, 1e-12))) * math.cos(2.0 * math.pi * u2)
    return int(min(hi, max(lo, round(median * math.exp(sigma * z)))))


def sphere_job_case(n: int, storage_les: bool = True) -> W.Case:
    """D3Q19 sphere channel of n^3 nodes: sphere radius 3n/32 at (n/4, n/2, n/2), the proportions of the
    256x128x128 sphere channel (radius 12 at x = 64 of 256, height 128)."""
    r = 3.0 * n / 32.0
    return W.sphere_channel(nx=n, ny=n, nz=n, radius=r, center=(n / 4.0, n / 2.0, n / 2.0), les=storage_les,
                            device_geometry=True)


def thermal_job_case(nx: int, rayleigh: float, seed: int) -> W.Case:
    """Rayleigh-Benard cell nx x nx/2, Pr = 0.71 (D2Q9 flow + D2Q5 temperature), TRT + Smagorinsky."""
    ny = nx // 2
    return W.rayleigh_benard(nx, ny, rayleigh, 0.71, u_free_fall=W.rb_free_fall_velocity(ny, rayleigh), seed=seed)


def mixed_jobs(n_jobs: int, rate: float, seed: int = W.BASE_SEED, d3q19_frac: float = 0.5,
               n_range=(48, 160), nx_range=(64, 512), median_steps: float = 2000.0, p5_steps: float = 500.0,
               steps_range=(200, 20000), thermal_frac: float = 0.1, ra_range=(1e4, 1e6)) -> list:
    """Poisson arrivals at `rate` jobs/s of D2Q9 jobs and D3Q19 sphere jobs (n^3, n ~ U[n_range]);
    steps lognormal (median 2000, 5th percentile 500, clipped). A D2Q9 job is a Rayleigh-Benard cell
    (NX ~ U[nx_range], NY = NX/2, Ra log-uniform in ra_range, Pr = 0.71) with probability
    thermal_frac, else a channel of the ellipse sweep. Job j draws its inter-arrival time, kind, size,
    steps and Ra from SplitMix64(seed + 1_000_000 + j)."""
    jobs, t = [], 0.0
    for j in range(n_jobs):
        u = W.uniform24(seed + 1_000_000 + j, 7).astype(np.float64)
        t += -math.log(max(1.0 - u[0], 1e-12)) / rate
        steps = lognormal_steps(u[1], u[2], median_steps, p5_steps, *steps_range)
        if u[3] < d3q19_frac:
            n = int(n_range[0] + math.floor(u[4] * (n_range[1] - n_range[0] + 1)))
            jobs.append(Job(j, "d3q19", (19, n, n, n), (lambda n=n: sphere_job_case(n)), steps, t, (1, True, 0.17)))
        elif u[5] < thermal_frac:
            nx = int(nx_range[0] + math.floor(u[4] * (nx_range[1] - nx_range[0] + 1)))
            ra = ra_range[0] * (ra_range[1] / ra_range[0]) ** u[6]
            make = (lambda nx=nx, ra=ra, j=j: thermal_job_case(nx, ra, seed + j))
            jobs.append(Job(j, "thermal", (9, nx, nx // 2, 1), make, steps, t, (1, True, 0.17)))
        else:
            nx = W.ellipse_sweep_dims(j, nx_range=nx_range, seed=seed)
            make = (lambda j=j: W.ellipse_sweep(1, nx_range=nx_range, seed=seed, first=j)[0])
            jobs.append(Job(j, "d2q9", (9, nx, nx // 2, 1), make, steps, t, (1, True, 0.17)))
    return jobs


def job_bytes(job: Job, storage: str) -> int:
    q, nx, ny, nz = job.dims
    flags = 2 if job.kind == "thermal" else 0  # bit 1: the coupled temperature's buffers
    return int(lib.wake_grid_estimate_bytes(q, nx, ny, nz, STORAGE[storage], flags))


# Sphere jobs at least this wide step alone through the single-lattice kernels (with CUDA graphs
# of SOLO_GRAPH_STEPS steps): measured on one B200 (FP32, TRT + LES), n = 112..160 run at 24-29k
# MLUPS alone, within 10% of a batch of equal jobs or faster, while smaller jobs gain 1.3-2.3x from
# batching (device rates measured by bench.py serving_rates). Solo jobs keep the batch's row lists
# short, and those lists are rebuilt whenever the batch's membership changes.
SOLO_MIN_EDGE = 112
SOLO_GRAPH_STEPS = 20


def _class_key(job: Job):
    if job.kind == "d3q19" and job.dims[1] >= SOLO_MIN_EDGE:
        return ("solo", job.id)
    return (job.dims[0],) + tuple(job.model)


class _Solo:
    """A job large enough to fill the device by itself, stepped through its own grid on its own
    stream (the batch interface the serving loop uses)."""

    def __init__(self):
        self.g = None
        self.case = None

    def set_stream(self, stream) -> None:
        self.stream = stream

    def use_graph(self, steps: int) -> None:
        self.graph = steps

    def add(self, g, collision, use_les=False, smag_const=0.14) -> None:
        self.g, self.model = g, (collision, use_les, smag_const)
        g.set_stream(self.stream)
        g.use_graph(SOLO_GRAPH_STEPS)

    def step(self, n: int) -> None:
        c, les, cs = self.model
        self.g.step(c, use_les=les, smag_const=cs, n=n)

    def remove(self, g) -> None:
        self.g = None

    def host_seconds(self) -> dict:
        return {}

    def close(self) -> None:
        self.g = None


def _start(job: Job, storage: str):
    """Resident lattice of a job; the force ring (65,536 entries) holds every step of the longest job."""
    case = job.make()
    return W.build_grid(case, storage=storage), case


def _finish(job: Job, g, arrival, admitted, now, error=None) -> JobResult:
    forces = np.zeros((0, 3))
    diag = (math.nan, math.nan, math.nan)
    nusselt = None
    if error is None:
        try:
            g.synchronize()
            forces = g.force_history()
            diag = g._diag()
            if job.kind == "thermal":
                nusselt = g.compute_nusselt_number()
        except Exception as e:  # a job that went non-finite reports its error, the others carry on
            error = str(e)
    return JobResult(job.id, job.kind, job.steps, arrival, admitted, now, forces, diag, error, job.nodes, nusselt)


# ------------------------------------------------------------------ server
class Server:
    """Admission by HBM budget and slots, continuous batching per job kind.

    Batches step with plain launches by default (graph_steps = 0). Membership changes at
    most ticks, and each change would re-capture a graph: on the mixed workload that
    capture was most of the loop's host time and made no tick shorter, because the device
    is the bottleneck there."""

    def __init__(self, budget_bytes: int, storage: str = "f32", max_tick_steps: int = 100, max_slots: int = 4096,
                 graph_steps: int = 0):
        self.budget = int(budget_bytes)
        self.storage = storage
        self.max_tick = max_tick_steps
        self.max_slots = max_slots
        self.graph_steps = graph_steps

    def run(self, jobs: list, realtime: bool = True, clock=time.perf_counter) -> ServeReport:
        import torch

        pending = collections.deque(sorted(jobs, key=lambda j: (j.arrival, j.id)))
        batches: dict = {}   # class key -> (Batch, torch stream)
        resident: dict = {}  # job id -> [job, grid, remaining, bytes, admitted, key]
        used = peak = 0
        results, ticks = [], 0
        t0 = clock()

        def now():
            return clock() - t0 if realtime else float(ticks)

        staged = []  # admitted and set up, joining their batch after the running tick
        phase = collections.defaultdict(float)  # host seconds per phase of the loop

        class _Timed:
            def __init__(self, name):
                self.name = name

            def __enter__(self):
                self.t = clock()

            def __exit__(self, *exc):
                phase[self.name] += clock() - self.t

        def admit():
            nonlocal used, peak
            while pending and (pending[0].arrival <= now() or not realtime):
                job = pending[0]
                need = job_bytes(job, self.storage)
                if need > self.budget:
                    pending.popleft()
                    results.append(_finish(job, None, job.arrival, now(), now(), error="larger than the HBM budget"))
                    continue
                if used + need > self.budget or len(resident) + len(staged) >= self.max_slots:
                    break
                pending.popleft()
                g, case = _start(job, self.storage)
                g._apply_model(case.collision, case.les, case.cs_smag)
                # flags, row lists and the initial collide on the job's own stream, then free the
                # FP32 start-up scratch: all of it overlaps the batches' running tick
                check(lib.wake_grid_release_scratch(g.handle))
                staged.append((job, g, case, need, now()))
                used += need
                peak = max(peak, used)

        while pending or resident or staged:
            # one tick: every batch advances by the steps its closest-to-done member needs
            advanced = {}
            with _Timed("launch"):
                for key, (b, _) in batches.items():
                    rem = [v[2] for v in resident.values() if v[5] == key]
                    if rem:
                        n = min(self.max_tick, min(rem))
                        b.step(n)
                        advanced[key] = n
            with _Timed("admit"):
                admit()  # host work of new arrivals while the tick runs
            with _Timed("wait"):
                for key in advanced:
                    torch.cuda.Stream.synchronize(batches[key][1])
            if advanced:
                ticks += 1
            t_now = now()
            for jid in list(resident):
                job, g, rem, need, adm, key = resident[jid]
                rem -= advanced.get(key, 0)
                resident[jid][2] = rem
                if rem <= 0:
                    with _Timed("finish"):
                        results.append(_finish(job, g, job.arrival, adm, t_now))
                        batches[key][0].remove(g)
                        g.close()
                        if key[0] == "solo":
                            batches.pop(key)[0].close()
                    used -= need
                    del resident[jid]
            for job, g, case, need, adm in staged:
                key = _class_key(job)
                if key not in batches:
                    b = _Solo() if key[0] == "solo" else Batch(job.dims[0], self.storage)
                    st = torch.cuda.Stream()
                    b.set_stream(st.cuda_stream)
                    b.use_graph(self.graph_steps)
                    batches[key] = (b, st)
                batches[key][0].add(g, case.collision, use_les=case.les, smag_const=case.cs_smag)
                resident[job.id] = [job, g, job.steps, need, adm, key]
            staged.clear()
            if not resident and pending and realtime:
                admit()
                if not staged:
                    time.sleep(max(0.0, min(0.005, pending[0].arrival - now())))
        makespan = now()
        inside = {"prepare": 0.0, "capture": 0.0, "launch": 0.0}
        for b, _ in batches.values():
            for k, v in b.host_seconds().items():
                inside[k] += v
            b.close()
        results.sort(key=lambda r: r.id)
        return ServeReport(results, makespan, ticks, peak, self.budget,
                           {"host_seconds": {k: round(v, 4) for k, v in phase.items()},
                            "batch_step_host_seconds": {k: round(v, 4) for k, v in inside.items()}})


def run_alone(job: Job, storage: str = "f32", graph_steps: int = 0) -> JobResult:
    """The job by itself through its own grid (no batch): the reference point of the mix."""
    g, c = _start(job, storage)
    if graph_steps:
        g.use_graph(graph_steps)
    g.step(c.collision, use_les=c.les, smag_const=c.cs_smag, n=job.steps)
    r = _finish(job, g, 0.0, 0.0, 0.0)
    g.close()
    return r


def run_per_job(jobs: list, storage: str = "f32", realtime: bool = True, clock=time.perf_counter) -> ServeReport:
    """Baseline: one job at a time in arrival order through its own grid with plain launches."""
    pending = sorted(jobs, key=lambda j: (j.arrival, j.id))
    results = []
    t0 = clock()
    for job in pending:
        if realtime:
            wait = job.arrival - (clock() - t0)
            if wait > 0:
                time.sleep(wait)
        adm = clock() - t0
        g, c = _start(job, storage)
        g.step(c.collision, use_les=c.les, smag_const=c.cs_smag, n=job.steps)
        results.append(_finish(job, g, job.arrival, adm, clock() - t0))
        g.close()
    return ServeReport(results, clock() - t0, len(pending), 0, 0)
