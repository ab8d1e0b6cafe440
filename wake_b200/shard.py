"""Independent work spread over ranks, one process per GPU, with no data-path collective.

A single lattice of the benchmark sizes fits one GPU, so several GPUs run
replicas of it. Batched sweeps and served job streams split by job instead.
Rank r takes jobs r, r + N, ... and runs them on its own GPU. Ranks meet only to
combine their timings and results: the maximum of their times, and the union of
their per-job results. Those exchanges run over the process group that
``torch.distributed`` was initialised with (NCCL on GPUs, gloo on the host).
"""
from __future__ import annotations

import numpy as np


def shard(items: list, rank: int, world: int) -> list:
    """Items rank, rank + world, rank + 2 world, ... (all of them for world = 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(items[rank::world])


class Ranks:
    """The process group's rank, size and the few collectives the benchmark needs; a
    one-process stand-in when torch.distributed is not initialised."""

    def __init__(self):
        import torch.distributed as dist

        self.on = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank() if self.on else 0
        self.world = dist.get_world_size() if self.on else 1
        self.backend = dist.get_backend() if self.on else None

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.on and self.world > 1:
            import torch.distributed as dist

            dist.barrier()

    def max(self, v: float) -> float:
        """The largest v over all ranks (each rank passes its own)."""
        if not self.on or self.world == 1:
            return float(v)
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(v)], dtype=torch.float64, device=self._device())
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if not self.on or self.world == 1:
            return float(v)
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(v)], dtype=torch.float64, device=self._device())
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def gather(self, obj) -> list:
        """Every rank's obj, in rank order, on every rank."""
        if not self.on or self.world == 1:
            return [obj]
        import torch.distributed as dist

        out = [None] * self.world
        dist.all_gather_object(out, obj)
        return out


def merge_served(parts: list) -> dict:
    """Combine per-rank served-run records into one whole-job summary.

    Each part holds ``jobs``, ``failed``, ``makespan_s``, ``node_steps`` and the list
    ``latencies_s`` of that rank's jobs. Ranks serve their shares at the same time, so
    the run's makespan is the largest one; sims/s counts every rank's jobs over it, and
    the latency percentiles are over all jobs."""
    lat = np.concatenate([np.asarray(p["latencies_s"], np.float64) for p in parts]) if parts else np.zeros(0)
    if lat.size == 0:
        lat = np.zeros(1)
    makespan = max(p["makespan_s"] for p in parts)
    jobs = sum(p["jobs"] for p in parts)
    return {"jobs": jobs, "failed": sum(p["failed"] for p in parts),
            "sims_per_s": jobs / makespan if makespan > 0 else 0.0,
            "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
            "mean_latency_s": float(lat.mean()), "makespan_s": makespan,
            "node_steps": int(sum(p["node_steps"] for p in parts)), "ranks": len(parts)}
