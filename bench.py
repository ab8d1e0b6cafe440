#!/usr/bin/env python3
"""Benchmark of the fused lattice update on the D3Q19 sphere channel.

Workload (one step = one time step of the whole lattice): D3Q19, 256x128x128,
TRT (Lambda = 1/4) + Smagorinsky LES (Cs = 0.17) applied per node, tau0 = 0.52,
sphere R = 12 at (64,64,64) with BFL curved links, Zou-He velocity inlet
u = 0.05 and pressure outlet rho = 1, periodic y/z, in-kernel momentum
exchange every step. FP32 populations; an FP16-storage leg runs the same
workload. Seeded synthetic inputs (no dataset).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl wake|reference]

N > 1 runs under torchrun: each rank advances its own replica of the sphere
channel and of the Taylor-Green cube, and takes its share (job id mod N) of the
batched sweep and of the served jobs. There is no data-path collective; timing is
the max over ranks of the CUDA-event time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FALLBACK_HBM_GBS = 6650.0
KERNEL_TIMING_STEPS = 200
WORKLOAD = ("D3Q19 TRT(Lambda=1/4)+Smagorinsky(Cs=0.17, applied) tau0=0.52, sphere R=12 at (64,64,64) with BFL "
            "links, Zou-He inlet u=0.05 / outlet rho=1, periodic y/z, in-kernel momentum exchange, 256x128x128")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4000)
    p.add_argument("--warmup", type=int, default=50)
    p.add_argument("--impl", choices=["wake", "reference"], default="wake")
    p.add_argument("--no-fp16", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-batch", action="store_true", help="skip the batched ellipse-sweep leg")
    p.add_argument("--batch-only", action="store_true", help="only the batched ellipse-sweep leg (one JSON line)")
    p.add_argument("--batch-steps", type=int, default=0,
                   help="with --batch-only: time this many steps instead of 5000 (a short run for ncu)")
    p.add_argument("--no-serve", action="store_true", help="skip the served-mix leg")
    p.add_argument("--no-tgv", action="store_true", help="skip the D3Q27 MRT Taylor-Green 384^3 leg")
    p.add_argument("--tgv-steps", type=int, default=5000, help="steps of the Taylor-Green leg (multiple of 500)")
    p.add_argument("--tgv-only", action="store_true", help="only the Taylor-Green leg (one JSON line)")
    p.add_argument("--tgv-size", type=int, default=384, help="edge of the Taylor-Green cube (384 = the workload)")
    p.add_argument("--serve-rate", type=float, default=200.0, help="arrival rate of the served-mix leg (jobs/s)")
    p.add_argument("--serve-jobs", type=int, default=1000,
                   help="jobs in the served-mix leg (latency percentiles over all of them)")
    p.add_argument("--serve-d3q19-frac", type=float, default=0.5,
                   help="with --serve-sweep: share of D3Q19 sphere jobs in the mix (0.5 = the workload)")
    p.add_argument("--serve-graph", type=int, default=0, help="steps per CUDA graph inside a served batch (0: plain)")
    p.add_argument("--serve-sweep", default=None,
                   help="comma-separated arrival rates: only the served mix at each rate (one JSON line per rate)")
    p.add_argument("--graph", type=int, default=20, help="steps per captured CUDA graph (0: plain launches)")
    p.add_argument("--profile", choices=["f32", "f16", "bf16", "f16c", "vorticity"], default=None,
                   help="profiling mode: only warm-up + timed steps of this storage, plain launches, one JSON line "
                        "('vorticity': --steps calls of the 3D vorticity / Q-criterion kernel on 256^3 device fields)")
    p.add_argument("--block", type=int, default=0, help="threads per block of the fused step (0: automatic)")
    p.add_argument("--kernel", type=int, default=0,
                   help="pure-gather kernel: 0 auto, 1 spans, 2 staged tiles, 3 whole rows, 4 pipelined whole rows")
    return p.parse_args()


def run_vorticity_profile(args, L=256):
    """Small command for ncu: the 3D vorticity / Q-criterion drop-in on device fields of L^3 nodes
    (three 67 MB inputs, four 67 MB outputs at L = 256: larger than L2)."""
    import torch

    import wake_b200 as wb
    from wake_b200 import workloads as W

    u = W.taylor_green_fields_device(L, 0.04)[1:]
    out = torch.empty((4, L ** 3), dtype=torch.float32, device="cuda")
    times = []
    for i in range(args.warmup + args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        wb.lib.compute_vorticity_and_q_criterion_3d(*[a.data_ptr() for a in u], *[o.data_ptr() for o in out], L, L, L)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        if i >= args.warmup:
            times.append(e0.elapsed_time(e1))
    ms = statistics.median(times) if times else float("nan")
    print(json.dumps({"profile": "vorticity", "nodes": L ** 3, "calls": args.steps, "ms_per_call": ms,
                      "achieved_gbs": 28 * L ** 3 / (ms * 1e-3) / 1e9}))


def run_profile(args):
    """Small command for ncu: the workload's fused step, nothing else."""
    import torch

    from wake_b200 import workloads as W

    import wake_b200 as wb

    if args.profile == "vorticity":
        run_vorticity_profile(args)
        return

    case = W.sphere_channel()
    g = W.build_grid(case, storage=args.profile)
    if args.block:
        wb.check(wb.lib.wake_grid_set_block(g.handle, args.block))
    wb.check(wb.lib.wake_grid_set_kernel(g.handle, args.kernel))
    if args.graph:
        g.use_graph(args.graph)
    ms = timed_steps(g, case, args.steps, args.warmup, 1)
    print(json.dumps({"profile": args.profile, "kernel": wb.lib.wake_grid_get_kernel(g.handle),
                      "block": wb.lib.wake_grid_get_block(g.handle), "steps": args.steps,
                      "ms_per_step": ms / args.steps, "mlups": case.n * args.steps / (ms * 1e-3) / 1e6}))
    torch.cuda.synchronize()


def hbm_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        try:
            return float(json.loads(f.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


KERNEL_NAMES = {1: ("wk::k_step_fast<19, TRT, {S}, LES, IDX32>", "spans"), 3: ("wk::k_step_rows<19, {S}, LES>", "rows"),
                4: ("wk::k_step_rows_pipe<19, {S}, LES, 256>", "pipe")}


def bulk_bytes_per_node(g, storage):
    """Algorithmic DRAM bytes per node of the D3Q19 bulk launch: 19 populations read and 19
    written, plus the node's flag byte for the span and tile kernels (variants 1, 2); the
    whole-row kernels read one descriptor byte per row instead (under 0.01 B per node)."""
    import wake_b200 as wb

    flag = 1 if wb.lib.wake_grid_get_kernel(g.handle) in (1, 2) else 0
    return 2 * 19 * (4 if storage == "f32" else 2) + flag


def bulk_kernel(g, storage):
    """(name, key of profiles/traffic.json) of the bulk kernel a grid steps with."""
    import wake_b200 as wb

    name, tag = KERNEL_NAMES.get(wb.lib.wake_grid_get_kernel(g.handle), ("unknown", "unknown"))
    return name.format(S=storage.upper()), f"d3q19_{storage}_{tag}"


def traffic_per_launch(key):
    """DRAM bytes (read + write) of one launch of a bulk kernel from the committed ncu capture
    (profiles/traffic.json): not measured in this run; (bytes, source) or (None, None)."""
    f = ROOT / "profiles" / "traffic.json"
    try:
        d = json.loads(f.read_text())
        e = d.get(key)
        if isinstance(e, dict):
            return e["bytes"], "ncu capture committed in profiles/traffic.json: " + d["_source"]
    except Exception:
        pass
    return None, None


class Clocks:
    """nvidia-smi sampler (200 ms) running across the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.samples = []
        self.proc = None
        self.gpu_id = gpu_id
        self.window = (0.0, 0.0)

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        threading.Thread(target=self._read, daemon=True).start()

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.time(), [x.strip() for x in line.split(",")]))

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        t0, t1 = self.window
        rows = [r for (t, r) in self.samples if t0 - 0.25 <= t <= t1 + 0.25] or [r for _, r in self.samples]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[0]) for r in rows if num(r[0]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 4 + i and r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][1]),
                "power_w_max": max((num(r[2]) or 0.0) for r in rows), "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        # NCCL between GPUs; gloo where no GPU is visible (host-side runs of the same logic)
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        from wake_b200.shard import Ranks

        Ranks().barrier()


def allmax(world, v):
    if world == 1:
        return v
    from wake_b200.shard import Ranks

    return Ranks().max(v)


def timed_steps(g, case, steps, warmup, world):
    import torch

    stream = torch.cuda.Stream()  # a real stream handle: the legacy default stream is 0
    g.set_stream(stream.cuda_stream)
    g.step(case.collision, use_les=case.les, smag_const=case.cs_smag, n=warmup)
    # the step graph (if any) is captured and instantiated here, outside the timed region
    g.prepare_steps(case.collision, use_les=case.les, smag_const=case.cs_smag)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    g.step(case.collision, use_les=case.les, smag_const=case.cs_smag, n=steps)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    g.synchronize()
    return allmax(world, start.elapsed_time(end))


def bulk_kernel_time(g, case, steps):
    """Average CUDA-event duration of the pure-gather (bulk) launch over `steps` plain steps.

    Events are recorded on the grid's stream around each bulk launch; the
    general-row launch runs concurrently on the forked stream, as in every step.
    Returns (ms per launch, nodes per launch)."""
    import ctypes

    import wake_b200 as wb

    wb.check(wb.lib.wake_grid_time_bulk_launches(g.handle, 1))
    g.step(case.collision, use_les=case.les, smag_const=case.cs_smag, n=steps)
    tot, cnt, nodes = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
    wb.check(wb.lib.wake_grid_bulk_launch_times(g.handle, ctypes.byref(tot), ctypes.byref(cnt), ctypes.byref(nodes)))
    wb.check(wb.lib.wake_grid_time_bulk_launches(g.handle, 0))
    g.synchronize()
    return tot.value / max(1, cnt.value), nodes.value


def storage_accuracy_c2(storage):
    """The C2 sphere channel at full size and length (2000 steps) in the form the reference can
    run, stored as `storage`, against the FP64 oracle's run of the same case kept in
    tests/golden/c2_sphere3d_trt.npz: velocity relative L2 on the planes z = 64 and y = 64 (every
    other node) and the drag coefficient (relative L2 of the history, and the relative error of the
    mean of the last 500 steps)."""
    import wake_b200 as wb  # noqa: F401
    from wake_b200 import workloads as W

    fx = ROOT / "tests" / "golden" / "c2_sphere3d_trt.npz"
    if not fx.exists():
        return None
    d = np.load(fx)
    steps = int(d["steps"])
    c = W.sphere_channel(reference_variant=True, collision=1, les=False)
    g = W.build_grid(c, storage=storage)
    g.use_graph(20)
    g.step(c.collision, use_les=False, n=steps)
    g.synchronize()
    m = g.macro()
    hist = g.force_history()
    g.close()
    q = 0.5 * 0.05 ** 2 * math.pi * 12.0 ** 2
    cd, cd64 = hist[:, 0] / q, d["forces_fp64"][:, 0].astype(np.float64) / q
    got, ref = [], []
    for k in ("ux", "uy", "uz"):
        a = m[k].reshape(c.nz, c.ny, c.nx)
        got.append(np.concatenate([a[64][::2, ::2].ravel(), a[:, 64, :][::2, ::2].ravel()]).astype(np.float64))
        ref.append(np.concatenate([d[f"fp64_{k}_z64"].ravel(), d[f"fp64_{k}_y64"].ravel()]).astype(np.float64))
    got, ref = np.concatenate(got), np.concatenate(ref)
    return {"case": "C2 sphere channel 256x128x128, 2000 steps, reference form (x-periodic, y/z walls, no Zou-He, "
                    "LES not applied), against the FP64 oracle", "storage": storage,
            "u_rel_l2": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "cd_history_rel_l2": float(np.linalg.norm(cd - cd64) / np.linalg.norm(cd64)),
            "cd_last500_rel": float(abs(cd[-500:].mean() - cd64[-500:].mean()) / abs(cd64[-500:].mean()))}


BATCH_WORKLOAD = ("batched D2Q9 TRT(Lambda=1/4)+Smagorinsky(Cs=0.17) ellipse sweep: 512 domains, NX~U[64,512], NY=NX/2, semi-axes in [NY/16,NY/6], "
                  "aspect in [1,3], angle of attack in [0,20] deg, Re in [50,300], inlet u=0.05, 5000 steps each")
STEPS_PER_SIM = 5000


def batched_leg(storage, n_domains=512, steps=STEPS_PER_SIM, warmup=20, baseline_jobs=16):
    """Sims/s of the ellipse sweep advanced as one batch, and of the same jobs launched per job.

    Batched: every domain resident, one bulk + one general launch + one force
    reduction per step for all 512 domains, CUDA graphs of 20 steps, bulk block
    size from the autotuner. Per job: the first `baseline_jobs` domains run one
    after another through their own grid with plain launches (the single-lattice
    API used once per job). Both time `steps` steps with CUDA events after warm-up;
    setup is outside both timed regions."""
    import torch

    import wake_b200 as wb
    from wake_b200 import workloads as W
    from wake_b200.batch import Batch

    from wake_b200.shard import Ranks, shard

    ranks = Ranks()
    all_cases = W.ellipse_sweep(n_domains)
    nodes = sum(c.n for c in all_cases)
    cases = shard(all_cases, ranks.rank, ranks.world)  # N GPUs: each batches its share of the sweep
    stream = torch.cuda.Stream()
    b = Batch(9, storage)
    b.set_stream(stream.cuda_stream)
    grids = []
    for c in cases:
        g = W.build_grid(c, storage=storage)
        b.add(g, c.collision, use_les=c.les, smag_const=c.cs_smag)
        grids.append(g)
    b.step(1)
    b.synchronize()
    for g in grids:
        wb.check(wb.lib.wake_grid_release_scratch(g.handle))
    best = b.autotune(steps=10)
    b.use_graph(20)
    b.step(warmup)
    torch.cuda.synchronize()
    ranks.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    b.step(steps)
    t1.record(stream)
    t1.synchronize()
    ms = ranks.max(t0.elapsed_time(t1))
    info = b.info()
    unstable = 0
    for g in grids:
        try:
            g.synchronize()
        except wb.WakeError:
            unstable += 1
    unstable = int(ranks.sum(unstable))
    b.close()
    for g in grids:
        g.close()
    del grids
    torch.cuda.synchronize()
    torch.cuda.empty_cache()

    # per-job plain launches on the same jobs' first `baseline_jobs` domains (shared out over the ranks)
    per_job_ms = 0.0
    base_nodes = 0
    ranks.barrier()
    for c in shard(all_cases[:baseline_jobs], ranks.rank, ranks.world):
        g = W.build_grid(c, storage=storage)
        g.set_stream(stream.cuda_stream)
        g.step(c.collision, use_les=c.les, smag_const=c.cs_smag, n=warmup)
        g.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(c.collision, use_les=c.les, smag_const=c.cs_smag, n=steps)
        e1.record(stream)
        e1.synchronize()
        per_job_ms += e0.elapsed_time(e1)
        base_nodes += c.n
        g.close()
    per_job_ms = ranks.max(per_job_ms)
    base_nodes = int(ranks.sum(base_nodes))
    bpn = 2 * 9 * (4 if storage == "f32" else 2) + 1
    sims = n_domains * steps / STEPS_PER_SIM / (ms * 1e-3)
    base_sims = baseline_jobs * steps / STEPS_PER_SIM / (per_job_ms * 1e-3)
    return {"metric": "sims/s", "value": sims, "unit": "sims/s", "storage": storage, "domains": n_domains,
            "nodes": nodes, "steps": steps, "ms_per_step": ms / steps, "mlups": nodes * steps / (ms * 1e-3) / 1e6,
            "achieved_gbs": bpn * nodes * steps / (ms * 1e-3) / 1e9, "bytes_per_node": bpn,
            "bulk_block": best, "bulk_rows": info["bulk_rows"], "general_rows": info["general_rows"],
            "launches_per_step": info["launches_per_step"], "unstable_members": unstable, "ranks": ranks.world,
            "per_job_plain": {"value": base_sims, "unit": "sims/s", "jobs": baseline_jobs,
                              "mlups": base_nodes * steps / (per_job_ms * 1e-3) / 1e6},
            "speedup_vs_per_job": sims / base_sims}


SERVE_WORKLOAD = ("served mix: Poisson arrivals of D2Q9 channel jobs (ellipse sweep domains, TRT+LES) and D3Q19 "
                  "sphere jobs (n^3, n~U[48,160], TRT+LES), 50/50, steps lognormal (median 2000, p5 500, clipped "
                  "200-20000), admission by an HBM budget of 80% of free device memory")


def serving_rates(storage="f32", steps=200, edges=(48, 64, 80, 96, 112, 128, 144, 160)):
    """Device rates (MLUPS, CUDA events over `steps` plain steps after 20) of the served job kinds:
    a sphere job of edge n alone through its own grid and as a batch of k equal jobs (k n^3 about
    4.2 M nodes); 64 channel jobs of the sweep batched; 16 Rayleigh-Benard cells batched."""
    import torch

    from wake_b200 import serve as S
    from wake_b200 import workloads as W
    from wake_b200.batch import Batch

    stream = torch.cuda.Stream()

    def timed(step):
        step(20)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3

    def batched(cases):
        b = Batch(cases[0].q, storage)
        b.set_stream(stream.cuda_stream)
        grids = []
        for c in cases:
            g = W.build_grid(c, storage=storage)
            b.add(g, c.collision, use_les=c.les, smag_const=c.cs_smag)
            grids.append(g)
        sec = timed(b.step)
        b.close()
        for g in grids:
            g.close()
        return sum(c.n for c in cases) * steps / sec / 1e6

    out = {"sphere": {}}
    for n in edges:
        c = S.sphere_job_case(n)
        g = W.build_grid(c, storage=storage)
        g.set_stream(stream.cuda_stream)
        sec = timed(lambda k: g.step(c.collision, use_les=c.les, smag_const=c.cs_smag, n=k))
        g.close()
        k = max(1, int(round(4.2e6 / n ** 3)))
        out["sphere"][n] = {"alone": n ** 3 * steps / sec / 1e6, "batched": batched([c] * k), "batch_members": k}
    out["d2q9_batched"] = batched(W.ellipse_sweep(64))
    out["thermal_batched"] = batched([S.thermal_job_case(128 + 16 * i, 1e4 * 10 ** (i % 3), W.BASE_SEED + i)
                                      for i in range(16)])
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def serving_cap(jobs, rates):
    """Device-time lower bound of a job list: every job at the best measured rate of its kind and size
    (sphere edges between the measured ones take the nearer edge's rate). Returns (seconds,
    sims/s of that bound, or of the arrival span when the arrivals take longer)."""
    edges = sorted(rates["sphere"])
    t = 0.0
    for j in jobs:
        if j.kind == "d3q19":
            n = min(edges, key=lambda e: abs(e - j.dims[1]))
            r = max(rates["sphere"][n]["alone"], rates["sphere"][n]["batched"])
        elif j.kind == "thermal":
            r = rates["thermal_batched"]
        else:
            r = rates["d2q9_batched"]
        t += j.nodes * j.steps / (r * 1e6)
    span = max(j.arrival for j in jobs) if jobs else 0.0
    return t, len(jobs) / max(t, span, 1e-12)


def serving_leg(rate, n_jobs, storage="f32", baseline=True, graph_steps=0, d3q19_frac=0.5, rates=None):
    """Continuous batching (wake_b200.serve.Server) against one-job-at-a-time plain launches on the same
    arrival list, both in real time. sims/s = jobs / makespan; latency = completion - arrival."""
    import torch

    from wake_b200 import serve as S
    from wake_b200.shard import Ranks, merge_served, shard

    ranks = Ranks()

    def whole(rep):
        # N GPUs: each serves the jobs whose id is its rank mod N, on the same arrival clock
        summ = rep.summary()
        parts = ranks.gather({"jobs": summ["jobs"], "failed": summ["failed"], "makespan_s": rep.makespan,
                              "node_steps": summ["node_steps"], "latencies_s": [r.latency for r in rep.results]})
        if ranks.world > 1:
            summ.update(merge_served(parts))
        return summ

    jobs = shard(S.mixed_jobs(n_jobs, rate, d3q19_frac=d3q19_frac), ranks.rank, ranks.world)
    free, _ = torch.cuda.mem_get_info()
    budget = int(0.8 * free)
    ranks.barrier()
    rep = S.Server(budget, storage=storage, max_tick_steps=100, graph_steps=graph_steps).run(jobs, realtime=True)
    out = {"rate_jobs_per_s": rate, "storage": storage, "graph_steps": graph_steps, **whole(rep)}
    out["mlups"] = out["node_steps"] / max(out["makespan_s"], 1e-9) / 1e6
    if rates is not None and ranks.world == 1:
        t_cap, cap = serving_cap(jobs, rates)
        out["cap"] = {"device_seconds": t_cap, "sims_per_s": cap, "fraction": out["sims_per_s"] / cap,
                      "rule": "every job at the best measured rate of its kind and size (serving_rates), "
                              "or the arrival span when longer"}
    if baseline:
        torch.cuda.empty_cache()
        ranks.barrier()
        base = whole(S.run_per_job(jobs, storage=storage, realtime=True))
        out["per_job_plain"] = {k: base[k] for k in ("sims_per_s", "p50_latency_s", "p99_latency_s", "makespan_s",
                                                     "failed")}
        out["speedup_vs_per_job"] = out["sims_per_s"] / max(base["sims_per_s"], 1e-12)
    return out


TGV_WORKLOAD = ("D3Q27 MRT periodic Taylor-Green vortex 384^3, u0=0.04, tau=0.51, FP32 populations vs FP16 and "
                "BF16 shifted storage (FP32 arithmetic)")


def tgv_leg(L=384, steps=5000, every=500, graph=20):
    """The three storages of the Taylor-Green lattice advanced side by side in chunks of `every` steps.

    Per chunk and storage: CUDA-event time of the chunk (the first chunk is warm-up and untimed),
    FP64 kinetic energy, and the velocity relative L2 error of FP16/BF16 against FP32 at the same
    step. KE is also set against the linear viscous decay exp(-6 nu k^2 t) of this initial field
    (its Laplacian is -3 k^2 u); the vortex is nonlinear at Re = u0/(nu k) = 733, so that column is
    context, not a gate. The comparison with FP64 runs on the 96^3 cube of the committed FP64 oracle
    run (tgv_vs_fp64)."""
    import torch

    import wake_b200 as wb
    from wake_b200 import workloads as W

    u0, tau = 0.04, 0.51
    n = L ** 3
    fields = W.taylor_green_fields_device(L, u0)
    stream = torch.cuda.Stream()
    grids = {}
    for st in ("f32", "f16", "bf16", "f16c"):
        g = wb.LatticeGrid3DQ27(L, L, L, tau, storage=st)
        g.set_stream(stream.cuda_stream)
        g.initialize_fields(*fields)
        g.set_periodic_axes(True, True)
        if graph:
            g.use_graph(graph)
        grids[st] = g
    del fields
    nu = (tau - 0.5) / 3.0
    k = 2.0 * math.pi / L
    ke0 = {st: g.compute_total_kinetic_energy() for st, g in grids.items()}
    u = {st: torch.empty((3, n), dtype=torch.float32, device="cuda") for st in grids}
    ms = {st: 0.0 for st in grids}
    timed_steps_done = 0
    rows = []
    for c in range(steps // every):
        for st, g in grids.items():
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.step(wb.MRT, n=every)
            e1.record(stream)
            e1.synchronize()
            if c > 0:
                ms[st] += e0.elapsed_time(e1)
            g.synchronize()
            g.macroscopic_into(ux=u[st][0], uy=u[st][1], uz=u[st][2])
        if c > 0:
            timed_steps_done += every
        t = (c + 1) * every
        ref_norm = torch.linalg.vector_norm(u["f32"].double()).item()
        row = {"step": t, "ke_ratio_linear": math.exp(-6.0 * nu * k * k * t)}
        for st, g in grids.items():
            row[f"ke_ratio_{st}"] = g.compute_total_kinetic_energy() / ke0[st]
            if st != "f32":
                row[f"u_rel_l2_{st}_vs_f32"] = torch.linalg.vector_norm((u[st] - u["f32"]).double()).item() / ref_norm
        rows.append(row)
    out = {"workload": TGV_WORKLOAD.replace("384^3", f"{L}^3"), "nodes": n, "steps": steps, "timed_steps": timed_steps_done,
           "graph_steps": graph, "checkpoints": rows}
    peak, _ = hbm_peak()
    for st in grids:
        bpn = 2 * 27 * (4 if st == "f32" else 2) + 1
        sec = ms[st] * 1e-3
        mlups = n * timed_steps_done / sec / 1e6 if sec > 0 else None
        gbs = bpn * n * timed_steps_done / sec / 1e9 if sec > 0 else None
        out[st] = {"mlups": mlups, "ms_per_step": ms[st] / max(1, timed_steps_done), "bytes_per_node": bpn,
                   "achieved_gbs": gbs, "frac_of_measured_hbm": gbs / peak if gbs else None}
    if out["f32"]["mlups"]:
        for st in ("f16", "bf16", "f16c"):
            out[st]["speedup_vs_f32"] = out[st]["mlups"] / out["f32"]["mlups"]
    for g in grids.values():
        g.close()
    # vorticity + Q-criterion of the final FP32 velocity: the drop-in kernel with device buffers,
    # 12 B read + 16 B written per node; CUDA events around each call on the legacy stream it uses
    res = torch.empty((4, n), dtype=torch.float32, device="cuda")
    uf = u["f32"]
    ev = []
    for i in range(13):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(torch.cuda.default_stream())
        wb.lib.compute_vorticity_and_q_criterion_3d(uf[0].data_ptr(), uf[1].data_ptr(), uf[2].data_ptr(),
                                                    res[0].data_ptr(), res[1].data_ptr(), res[2].data_ptr(),
                                                    res[3].data_ptr(), L, L, L)
        e1.record(torch.cuda.default_stream())
        e1.synchronize()
        if i >= 3:
            ev.append(e0.elapsed_time(e1))
    ms_q = statistics.median(ev)
    out["vorticity_q"] = {"ms_per_call": ms_q, "bytes_per_node": 28, "achieved_gbs": 28 * n / (ms_q * 1e-3) / 1e9,
                          "frac_of_measured_hbm": 28 * n / (ms_q * 1e-3) / 1e9 / peak,
                          "timing": "median of 10 calls after 3, CUDA events around each synchronous call "
                                    "(includes the call's host overhead)"}
    del res, u
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    out["vs_fp64"] = tgv_vs_fp64()
    return out


def load_workloads():
    """wake_b200/workloads.py loaded by path: its case builders are numpy only, and importing the
    wake_b200 package would load libwake_b200.so into a process that must not use it."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("wake_workloads_np", ROOT / "wake_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # dataclasses look their module up while the file executes
    spec.loader.exec_module(mod)
    return mod


REFERENCE_VARIANT = ("the reference's own LatticeGrid3D::step + momentum exchange (oracle/_ref: its host classes and "
                     "its kernels translated mechanically from ISPC) on the same 256x128x128 sphere channel, TRT, "
                     "tau0=0.52, BFL links, momentum exchange every step, in the form the reference can express: "
                     "x-periodic, y/z half-way walls, no Zou-He (the reference has no 3D Zou-He), Smagorinsky tau "
                     "computed but not applied (the reference discards it)")


def tgv_vs_fp64(storages=("f32", "f16", "bf16", "f16c")):
    """The Taylor-Green case (D3Q27 MRT, u0 = 0.04, tau = 0.51) on the 96^3 cube of the committed FP64
    oracle run (tests/golden/c3_tgv96_mrt_fp64.npz), per storage: every 500 steps the velocity
    relative L2 error against FP64 (every third node in each direction) and the kinetic energy's
    relative error."""
    import wake_b200 as wb  # noqa: F401
    from wake_b200 import workloads as W

    fx = ROOT / "tests" / "golden" / "c3_tgv96_mrt_fp64.npz"
    if not fx.exists():
        return None
    d = np.load(fx)
    L, every, sub = int(d["edge"]), int(d["every"]), int(d["sub"])
    case = W.taylor_green(L=L, u0=0.04, tau=0.51, q=27, collision=2)
    out = {"case": f"D3Q27 MRT Taylor-Green {L}^3, u0=0.04, tau=0.51, {int(d['steps'])} steps, against the FP64 oracle"}
    for st in storages:
        g = W.build_grid(case, storage=st)
        rows = []
        for k in range(int(d["steps"]) // every):
            g.step(2, n=every)
            g.synchronize()
            m = g.macro()
            u = np.stack([m[a].reshape(L, L, L)[::sub, ::sub, ::sub] for a in ("ux", "uy", "uz")]).astype(np.float64)
            ref = d["u"][k].astype(np.float64)
            rows.append({"step": every * (k + 1), "u_rel_l2": float(np.linalg.norm(u - ref) / np.linalg.norm(ref)),
                         "ke_rel": float(g.compute_total_kinetic_energy() / float(d["ke"][k + 1]) - 1.0)})
        g.close()
        out[st] = rows
    return out


def reference_sample(case_ref, steps, warmup, budget_s, threads=1):
    """Time the reference's own LatticeGrid3D::step + momentum exchange (oracle/_ref) on host cores:
    `threads` independent replicas (the reference is single-threaded), `warmup` untimed steps each,
    then `steps` timed steps each, fewer if they would not fit `budget_s` at the warm-up's pace."""
    import oracle

    L = oracle.ref()
    if L is None:
        return None
    c = case_ref
    grids = []
    for _ in range(threads):
        gr = oracle.RefGrid3D(c.nx, c.ny, c.nz, c.tau)
        gr.init_fields(c.rho, c.ux, c.uy, c.uz)
        L.ref3d_set_periodic(gr._h, 1)
        L.ref3d_set_solid_sphere(gr._h, *c.sphere)
        L.ref3d_build_curved_sphere_links(gr._h, *c.sphere)
        grids.append(gr)

    def run(gr, n):
        gr.step_forces(n, c.collision, c.mem[:3], c.mem[3], use_les=True, cs=c.cs_smag)

    def parallel(n):
        ths = [threading.Thread(target=run, args=(gr, n)) for gr in grids]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        return time.perf_counter() - t0

    t_warm = parallel(max(1, warmup))
    t_step = t_warm / max(1, warmup)
    n = int(max(1, min(steps, budget_s // max(t_step, 1e-6))))
    dt = parallel(n)
    mlups = threads * c.n * n / dt / 1e6
    return {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "reference",
            "sample": f"{n} timed steps after {max(1, warmup)} untimed, on each of {threads} independent replica(s) "
                      f"of {REFERENCE_VARIANT}",
            "seconds": dt, "steps": n, "per_core_mlups": mlups / threads}


def workload_config(n_nodes, world):
    """The `config` of both arms' JSON lines (the workload, not run results)."""
    return {"workload": WORKLOAD, "nodes": n_nodes, "storage": "f32",
            "l2": "inputs larger than L2 (two 319 MB population buffers, 126 MB L2)",
            "parallelism": ("replicas of the sphere channel and the Taylor-Green cube; batched sweep and served jobs "
                            "split by job id mod N") if world > 1 else "single GPU"}


def run_reference_impl(args):
    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    W = load_workloads()
    c = W.sphere_channel(reference_variant=True, collision=1, les=False)
    try:
        import psutil

        mem_cap = int(psutil.virtual_memory().available // (1.5 * 2**30))
    except Exception:
        mem_cap = 4
    threads = max(1, min(os.cpu_count() or 1, 32, mem_cap))
    res = reference_sample(c, steps=max(1, args.steps), warmup=max(1, args.warmup), budget_s=120.0, threads=threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libwake_ref.so missing"}))
        return
    ms = res["seconds"] * 1e3 / res["steps"]
    line = {"impl": "reference", "metric": "MLUPS", "value": res["value"], "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": res["steps"], "warmup": max(1, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64; no dataset)",
            "config": workload_config(c.n, world),
            "reference_variant": REFERENCE_VARIANT,
            "per_core_mlups": res["per_core_mlups"],
            "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": res["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if res["steps"] < args.steps:
        line["steps_requested"] = args.steps
    print(json.dumps(line))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference_impl(args)
        return
    if args.profile:
        run_profile(args)
        return
    if args.serve_sweep:
        rates = serving_rates()
        print(json.dumps({"serving_rates_mlups": rates}), flush=True)
        for rate in [float(r) for r in args.serve_sweep.split(",")]:
            wl = SERVE_WORKLOAD if args.serve_d3q19_frac == 0.5 else \
                SERVE_WORKLOAD.replace("50/50", f"D3Q19 fraction {args.serve_d3q19_frac}")
            print(json.dumps({"workload": wl, **serving_leg(rate, args.serve_jobs, graph_steps=args.serve_graph,
                                                            d3q19_frac=args.serve_d3q19_frac, rates=rates)}),
                  flush=True)
        return
    if args.tgv_only:
        print(json.dumps(tgv_leg(L=args.tgv_size, steps=args.tgv_steps)))
        return
    if args.batch_only:
        # --batch-steps: a short run for profiling, with a proportionally short per-job baseline
        kw = {"steps": args.batch_steps, "baseline_jobs": 2} if args.batch_steps else {}
        out = {"workload": BATCH_WORKLOAD, "f32": batched_leg("f32", **kw), "f16": batched_leg("f16", **kw)}
        print(json.dumps(out))
        return
    world, rank, local = dist_setup(args)
    import torch

    import wake_b200 as wb
    from wake_b200 import workloads as W

    torch.cuda.set_device(local)
    dev_uuid = None
    try:
        dev_uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    case = W.sphere_channel()
    clocks = Clocks(dev_uuid)
    clocks.start()
    peak, peak_kind = hbm_peak()

    # ---- FP32 leg (headline)
    g = W.build_grid(case, storage="f32")
    if args.graph:
        g.use_graph(args.graph)
    t_begin = time.time()
    ms = timed_steps(g, case, args.steps, args.warmup, world)
    clocks.window = (t_begin, time.time())
    n_nodes = case.n
    ms_step = ms / args.steps
    value = world * n_nodes * args.steps / (ms * 1e-3) / 1e6
    launches_per_step = wb.check(wb.lib.wake_grid_launches_per_step(g.handle))
    bpn = bulk_bytes_per_node(g, "f32")
    k_ms, k_nodes = bulk_kernel_time(g, case, KERNEL_TIMING_STEPS)
    achieved = bpn * k_nodes / (k_ms * 1e-3) / 1e9
    kname, kkey = bulk_kernel(g, "f32")
    traffic, traffic_src = traffic_per_launch(kkey)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": f"{peak_kind} HBM copy bandwidth", "traffic": traffic, "traffic_source": traffic_src,
            "bytes_per_node": bpn, "kernel": kname,
            "launch_ms": k_ms, "nodes_per_launch": k_nodes,
            "timing": f"CUDA events around each bulk launch over {KERNEL_TIMING_STEPS} plain steps after the timed "
                      "region; achieved = bytes_per_node x nodes_per_launch / launch_ms",
            "whole_step_gbs": bpn * n_nodes / (ms_step * 1e-3) / 1e9}
    forces = g.force_history()
    del g
    torch.cuda.empty_cache()

    # ---- 16-bit storage legs: FP16 (the addition's format) and FP16C
    def storage_leg(st):
        g16 = W.build_grid(case, storage=st)
        if args.graph:
            g16.use_graph(args.graph)
        ms16 = timed_steps(g16, case, args.steps, args.warmup, world)
        bpn16 = bulk_bytes_per_node(g16, st)
        k16_ms, k16_nodes = bulk_kernel_time(g16, case, KERNEL_TIMING_STEPS)
        ach16 = bpn16 * k16_nodes / (k16_ms * 1e-3) / 1e9
        kname16, kkey16 = bulk_kernel(g16, st)
        traffic16, _ = traffic_per_launch(kkey16)
        leg = {"value": world * n_nodes * args.steps / (ms16 * 1e-3) / 1e6, "unit": "MLUPS",
               "ms_per_step": ms16 / args.steps, "speedup_vs_f32": ms / ms16,
               "roofline": {"achieved": ach16, "peak": peak, "frac": ach16 / peak, "bytes_per_node": bpn16,
                            "launch_ms": k16_ms, "kernel": kname16, "traffic": traffic16,
                            "traffic_source": "as roofline.traffic_source" if traffic16 else None}}
        del g16
        torch.cuda.empty_cache()
        return leg

    fp16 = None
    if not args.no_fp16:
        fp16 = storage_leg("f16")
        fp16["accuracy_vs_fp64"] = storage_accuracy_c2("f16")
        fp16["bf16_accuracy_vs_fp64"] = storage_accuracy_c2("bf16")
        fp16["f16c"] = storage_leg("f16c")
        fp16["f16c"]["format"] = ("FP16C of h = f/w - 1: 1 sign, 4 exponent, 11 mantissa bits (Lehmann et al., "
                                  "Phys. Rev. E 106, 015308, 2022), |h| < 2")
        fp16["f16c"]["accuracy_vs_fp64"] = storage_accuracy_c2("f16c")

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        g = W.build_grid(case, storage="f32")
        if args.graph:
            g.use_graph(args.graph)
        # the job's input: per-node initial fields in pinned host memory, as the reference's
        # LatticeGrid3D::initialize_custom takes them (the grid builds the equilibrium)
        fields = {k: torch.from_numpy(np.ascontiguousarray(getattr(case, k), np.float32)).pin_memory()
                  for k in ("rho", "ux", "uy", "uz")}
        out = {k: torch.empty(n_nodes, dtype=torch.float32).pin_memory() for k in ("rho", "ux", "uy", "uz", "speed")}

        def job(steps):
            wb.check(wb.lib.wake_grid_initialize_fields(g.handle, *[fields[k].data_ptr()
                                                                    for k in ("rho", "ux", "uy", "uz")]))
            g.step(case.collision, use_les=case.les, smag_const=case.cs_smag, n=steps)
            h = g.force_history()
            wb.check(wb.lib.wake_grid_get_macroscopic(g.handle, *[out[k].data_ptr() for k in ("rho", "ux", "uy",
                                                                                             "uz", "speed")]))
            return h

        job(max(args.warmup, 2 * max(args.graph, 1)))  # untimed: first-use costs (graph capture, copy paths)
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        hist = job(args.steps)
        dt = allmax(world, time.perf_counter() - t0)
        h2d = sum(v.numel() * 4 for v in fields.values())
        d2h = hist.nbytes + sum(v.numel() * 4 for v in out.values())
        e2e = {"value": world * n_nodes * args.steps / dt / 1e6, "unit": "MLUPS",
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "job": "H2D of the initial rho/u fields from pinned host memory (wake_grid_initialize_fields, "
                      "the reference's initialize_custom; equilibrium built on the device), K fused steps "
                      "through wake_grid_step, D2H of the per-step force history and of rho/u/speed; after "
                      "one untimed shorter job on the same grid; wall clock around the job"}
        del g
    batched = None
    if not args.no_batch:
        batched = {"workload": BATCH_WORKLOAD, "f32": batched_leg("f32"), "f16": batched_leg("f16")}
    tgv = None
    if not args.no_tgv:
        tgv = tgv_leg(L=args.tgv_size, steps=args.tgv_steps)
    served = None
    if not args.no_serve:
        rates = serving_rates() if world == 1 else None
        served = {"workload": SERVE_WORKLOAD, **serving_leg(args.serve_rate, args.serve_jobs,
                                                            graph_steps=args.serve_graph, rates=rates)}
        if rates is not None:
            served["device_rates_mlups"] = rates
    clocks.stop()

    # ---- CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        c_ref = W.sphere_channel(reference_variant=True, collision=1, les=False)
        res = reference_sample(c_ref, steps=40, warmup=1, budget_s=20.0, threads=1)
        if res is not None:
            cpu = {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        cd = forces[-1, 0] / (0.5 * 0.05 ** 2 * math.pi * 144.0) if len(forces) else None
        line = {"metric": "MLUPS", "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded SplitMix64; no dataset)",
                "config": workload_config(n_nodes, world), "graph_steps": args.graph, "final_cd": cd,
                "roofline": roof, "fp16": fp16, "cpu_baseline": cpu, "e2e": e2e, "batched": batched, "taylor_green": tgv, "served": served,
                "clocks": clocks.summary(),
                "gpu_launches": launches_per_step * args.steps}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
