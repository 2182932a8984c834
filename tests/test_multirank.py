"""The multi-GPU path's host logic with 2 gloo ranks on CPU: worlds are partitioned across ranks
(disjoint, complete, balanced, the same on every rank) and timing aggregates as the max over
ranks with events summed. The data path has no collective: worlds never exchange frames."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from twins_b200 import shard, workloads


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=size)
    worlds = workloads.c4(seed=3, n_worlds=12, min_flows=50, max_flows=400)
    mine = shard.shard(worlds, rank, size)
    gathered = [None] * size
    dist.all_gather_object(gathered, mine)
    ms, ev = shard.aggregate(10.0 * (rank + 1), 100.0 * (rank + 1), dist)
    out[rank] = (gathered, ms, ev)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_partition_and_aggregate():
    size, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_rank, args=(size, port, out), nprocs=size, start_method="spawn", join=True)
    g0, ms0, ev0 = out[0]
    g1, _, _ = out[1]
    assert g0 == g1  # every rank computes the same partition
    a, b = g0
    assert not set(a) & set(b) and sorted(a + b) == list(range(12))
    worlds = workloads.c4(seed=3, n_worlds=12, min_flows=50, max_flows=400)
    la, lb = (sum(shard.work_of(worlds[i]) for i in part) for part in (a, b))
    assert max(la, lb) <= 1.5 * min(la, lb)
    assert ms0 == 20.0 and ev0 == 300.0  # max of times, sum of events


def test_single_rank_is_identity():
    worlds = workloads.c1()
    assert shard.shard(worlds, 0, 1) == [0]
    assert shard.aggregate(5.0, 7.0) == (5.0, 7.0)
    with pytest.raises(ValueError):
        shard.shard(worlds, 2, 2)
