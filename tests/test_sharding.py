"""Multi-GPU host logic on the CPU: the instance partition every rank
computes for itself, and the bench's timing reductions, run as two gloo
ranks (world size 2).  Instances are independent, so the only collective
traffic is the barrier and the max / sum of per-rank timings."""
import importlib.util
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _load_bench():
    spec = importlib.util.spec_from_file_location("pcg_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_partition_covers_every_instance_once_and_balances(pcg):
    from pcg import sharding, workloads
    work = workloads.batched_3d_work(n_instances=128)
    for world in (1, 2, 3, 4, 8):
        parts = sharding.partition(work, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(128))
        loads = sharding.shard_loads(work, parts)
        # greedy packing: no shard exceeds the mean by more than one instance
        assert max(loads) <= sum(work) / world + max(work)
        assert sharding.partition(work, world) == parts          # deterministic
    with pytest.raises(ValueError):
        sharding.partition(work, 0)


def test_shard_builds_the_same_instances_as_the_full_set(pcg):
    import numpy as np
    from pcg import workloads
    full = workloads.batched_3d(n_instances=6, max_cells=3000)
    part = workloads.batched_3d(n_instances=6, max_cells=3000, only=[1, 4])
    assert np.array_equal(part[0].soa, full[1].soa) and np.array_equal(part[1].soa, full[4].soa)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    bench = _load_bench()
    bench.load_pcg()
    r, w, local, dist = bench.setup_dist(world, backend="gloo")
    try:
        shard = bench.rank_shard(64, r, w)
        shards = [None] * w
        dist.all_gather_object(shards, shard)
        t_max = bench.dist_max(dist, local, 1.0 + r)
        t_sum = bench.dist_sum(dist, local, 10.0 * (r + 1))
        bench.barrier(dist)
        with open(os.path.join(out_dir, f"rank{r}.txt"), "w") as f:
            f.write(repr((shards, t_max, t_sum)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_disjoint_shards_and_reduce_timings(pcg, tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    res = [eval(open(tmp_path / f"rank{r}.txt").read()) for r in range(world)]
    assert res[0] == res[1]                                   # same view on both ranks
    shards, t_max, t_sum = res[0]
    assert sorted(shards[0] + shards[1]) == list(range(128))
    assert not set(shards[0]) & set(shards[1])
    assert t_max == 2.0 and t_sum == 30.0
