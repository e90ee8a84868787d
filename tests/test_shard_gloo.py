"""Multi-GPU host logic on the CPU: two gloo ranks partition the batched
models identically without communicating, gather their per-model results to
rank 0, and take the slowest rank's time -- the same calls bench.py makes
over NCCL with one GPU per rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from artisynth_core_b200 import shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, weights, out_q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        parts = shard.lpt_partition(weights, world)
        mine = parts[rank]
        # stand-in for the rank's pack results: model index -> steps taken
        local = {i: 20 for i in mine}
        gathered = shard.gather_to_root(dist, {"rank": rank, "models": mine, "results": local})
        slowest = shard.max_over_ranks(dist, 1.0 + rank)
        if rank == 0:
            out_q.put((parts, gathered, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_lpt_partition_balances_and_covers():
    w = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = shard.lpt_partition(w, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(w)))
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(w)
    assert shard.lpt_partition(w, 3) == parts  # deterministic
    assert shard.lpt_partition(w, 1) == [list(range(len(w)))]
    with pytest.raises(ValueError):
        shard.lpt_partition(w, 0)


def test_two_gloo_ranks_partition_and_gather():
    weights = [float(100 + 37 * (i % 7)) for i in range(16)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, weights, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, gathered, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert parts == shard.lpt_partition(weights, 2)
    assert [g["rank"] for g in gathered] == [0, 1]
    assert sorted(sum((g["models"] for g in gathered), [])) == list(range(16))
    assert all(set(g["results"]) == set(g["models"]) for g in gathered)
    assert slowest == 2.0
