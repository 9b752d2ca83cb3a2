"""Multi-rank placement and reductions on CPU: two `gloo` ranks (the
one-process-per-GPU layout of bench.py and of sharded batched / served
runs) plan the same shards without communicating, cover every simulation
exactly once, and reduce their timings to the slowest rank's."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from galaxy_b200.shard import plan_shards, work_estimate


def test_plan_is_balanced_and_complete():
    rng = np.random.default_rng(3)
    sizes = [int(2 ** rng.uniform(10, 18)) for _ in range(512)]
    for world in (1, 2, 3, 8):
        shards = plan_shards(sizes, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(work_estimate(sizes[i]) for i in s) for s in shards]
        # LPT: no rank exceeds the mean by more than the largest single job
        assert max(loads) <= sum(loads) / world + max(work_estimate(n) for n in sizes)


def test_plan_respects_budget():
    sizes = [1000] * 10
    shards = plan_shards(sizes, 2, footprint=lambda i: 100, budget_bytes=500)
    assert sorted(len(s) for s in shards) == [5, 5]
    with pytest.raises(MemoryError):
        plan_shards(sizes, 2, footprint=lambda i: 100, budget_bytes=400)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, out_dir):
    import torch.distributed as dist

    from galaxy_b200.shard import gather_to_all, max_over_ranks, plan_shards, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shards = plan_shards(sizes, world)
        mine = shards[rank]
        # stand-in for the device work: particle-steps done and a rank time
        done = {i: sizes[i] * 3 for i in mine}
        ms = 10.0 + rank
        slowest = max_over_ranks(dist, ms)
        total = sum_over_ranks(dist, sum(done.values()))
        every = gather_to_all(dist, done)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as fh:
            fh.write(json.dumps([slowest, total, sorted(k for d in every for k in d)]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_cover_every_simulation_once(tmp_path):
    sizes = [1024 * (k + 1) for k in range(37)]
    mp.spawn(_rank_main, args=(2, _free_port(), sizes, str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        slowest, total, ids = json.loads(open(tmp_path / f"rank{r}.txt").read())
        assert slowest == 11.0
        assert total == 3.0 * sum(sizes)
        assert ids == list(range(len(sizes)))
