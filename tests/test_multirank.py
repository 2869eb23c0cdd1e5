"""CPU, world_size 2 over gloo: the multi-rank host logic of bench.py
(replica seeds, max-over-ranks device time, summed replica rates)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.over_ranks(10.0 + rank, "max", world, "cpu")
        r = bench.over_ranks(100.0 * (rank + 1), "sum", world, "cpu")
        out[rank] = (t, r, bench.replica_seed(2887, rank))
    finally:
        dist.destroy_process_group()


def test_two_rank_reductions_and_seeds():
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 11.0          # slowest replica
    assert res[0][1] == res[1][1] == 300.0         # total of the replicas' rates
    assert res[0][2] != res[1][2]                  # independent replicas


def test_single_process_passthrough():
    import bench
    assert bench.over_ranks(3.5, "max", 1, "cpu") == 3.5


def test_batch_shards_cover_every_instance_once_and_balance():
    import bench
    specs = bench.batch_specs(256)
    for world in (1, 2, 3, 8):
        shards = [bench.shard_instances(specs, world, r) for r in range(world)]
        flat = sorted(i for sh in shards for i in sh)
        assert flat == list(range(len(specs)))
        loads = [sum((2 * specs[i][2]) ** 2 for i in sh) for sh in shards]
        assert max(loads) <= min(loads) + max((2 * s[2]) ** 2 for s in specs)
    assert bench.shard_instances(specs, 1, 0) == list(range(len(specs)))
