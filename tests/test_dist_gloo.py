"""The multi-rank host logic on CPU with world size 2 over gloo: the timing
reduction of bench.py (max over ranks), and the round-robin sharding of batched
designs with the gather of their results (homo3d_b200/batch.py)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, check):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        if check == "max":
            import bench
            assert bench.max_over_ranks(dist, 10.0 + rank) == 10.0 + world - 1
            assert bench.max_over_ranks(None, 3.5) == 3.5
        else:
            from homo3d_b200.batch import gather_designs, max_over_ranks, shard
            n = 7
            mine = shard(n, rank, world)
            assert mine == list(range(rank, n, world))
            rows = gather_designs(dist, n, mine, [{"design": i, "rank": rank} for i in mine])
            assert [r["design"] for r in rows] == list(range(n))
            assert [r["rank"] for r in rows] == [i % world for i in range(n)]
            assert max_over_ranks(dist, [1.0 * rank, 5.0 - rank]) == [world - 1.0, 5.0]
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("check", ["max", "batch"])
def test_two_ranks_over_gloo(check):
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    mp.spawn(_worker, args=(2, _free_port(), check), nprocs=2, join=True)
