"""Multi-rank host logic on CPU (gloo, world size 2)."""
import importlib.util
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _replicas():
    spec = importlib.util.spec_from_file_location("pe_replicas", ROOT / "protein_encoding_v2_nsga-iii_b200" / "replicas.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rep = _replicas()
    t = rep.max_over_ranks(1.5 + rank)
    shards = rep.shard_jobs([5, 1, 9, 3, 3, 7], world)
    seed = rep.replica_seed(2024, rank)
    # end to end: each rank "runs" its shard of jobs and the results are gathered
    costs = [5, 1, 9, 3, 3, 7]
    mine = shards[rank]
    gathered = rep.gather_results({j: {"rank": rank, "cost": costs[j]} for j in mine})
    q.put((rank, t, shards, seed, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_timing_and_sharding():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(t == 2.5 for _, t, _, _, _ in res)              # max over ranks
    for _, _, shards_r, _, gathered in res:                    # every rank holds every job's result once
        assert sorted(gathered) == list(range(6))
        assert all(gathered[j]["rank"] == r for r, s in enumerate(shards_r) for j in s)
    assert res[0][2] == res[1][2]                              # same assignment on every rank
    shards = res[0][2]
    assert sorted(i for s in shards for i in s) == list(range(6))
    loads = [sum([5, 1, 9, 3, 3, 7][i] for i in s) for s in shards]
    assert max(loads) - min(loads) <= 2
    assert res[0][3] != res[1][3]                              # distinct replica seeds


def test_whole_job_rate():
    rep = _replicas()
    assert rep.whole_job_rate(20, 4, 2.0) == 40.0
