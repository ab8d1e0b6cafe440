"""Several ranks on the host (gloo, world size 2): the logic that spreads batched and served
jobs over GPUs and combines their timings, run without a GPU.

Each rank takes the jobs whose position is its rank mod N; ranks meet only to take the
maximum of their times and to gather their per-job results (wake_b200/shard.py, used by
bench.py under torchrun).
"""
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from wake_b200 import serve as S
    from wake_b200.shard import Ranks, merge_served, shard

    r = Ranks()
    res = {"rank": r.rank, "world": r.world, "backend": r.backend,
           "max": r.max(1.5 + rank), "sum": r.sum(1.0 + rank), "gather": r.gather(rank * 10),
           "bench_allmax": bench.allmax(world, 3.0 * rank)}
    bench.barrier(world)
    jobs = S.mixed_jobs(40, 100.0, n_range=(16, 24), nx_range=(64, 96))
    mine = shard(jobs, r.rank, r.world)
    res["ids"] = r.gather([j.id for j in mine])
    # a stand-in for this rank's served run: latency = steps / 1000 s, makespan by rank
    lat = [j.steps / 1000.0 for j in mine]
    part = {"jobs": len(mine), "failed": 0, "makespan_s": 2.0 + rank, "node_steps": sum(j.nodes * j.steps for j in mine),
            "latencies_s": lat}
    res["merged"] = merge_served(r.gather(part))
    res["all_latencies"] = [j.steps / 1000.0 for j in jobs]
    res["all_node_steps"] = sum(j.nodes * j.steps for j in jobs)
    (Path(out_dir) / f"rank{rank}.json").write_text(json.dumps(res))
    dist.barrier()
    dist.destroy_process_group()


def test_two_host_ranks_share_jobs_and_combine_results(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    out = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for r, o in enumerate(out):
        assert o["rank"] == r and o["world"] == world and o["backend"] == "gloo"
        assert o["max"] == 2.5 and o["sum"] == 3.0 and o["gather"] == [0, 10]
        assert o["bench_allmax"] == 3.0
        # the two shares are disjoint and cover every job
        ids = o["ids"]
        assert not set(ids[0]) & set(ids[1]) and sorted(ids[0] + ids[1]) == list(range(40))
        m = o["merged"]
        assert m["jobs"] == 40 and m["ranks"] == 2 and m["makespan_s"] == 3.0
        assert m["sims_per_s"] == pytest.approx(40 / 3.0)
        assert m["node_steps"] == o["all_node_steps"]
        assert m["p50_latency_s"] == pytest.approx(float(np.percentile(o["all_latencies"], 50)))
        assert m["p99_latency_s"] == pytest.approx(float(np.percentile(o["all_latencies"], 99)))


def test_shard_single_rank_is_identity():
    from wake_b200.shard import Ranks, shard

    assert shard(list(range(7)), 0, 1) == list(range(7))
    assert shard(list(range(7)), 1, 3) == [1, 4]
    with pytest.raises(ValueError):
        shard([1], 2, 2)
    r = Ranks()
    assert (r.rank, r.world) == (0, 1) and r.max(4.0) == 4.0 and r.gather("x") == ["x"]
