"""CPU: the replicated multi-GPU path's host logic with two gloo ranks (no GPU): the job time is
the max over ranks and the completed solves are summed, as bench.py aggregates an N-GPU run."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times, counts = bench.reduce_over_ranks(dist, [1.0 + rank, 10.0 * (world - rank)], [3 + rank], "cpu")
        out[rank] = (times, counts)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_reduce_over_ranks_gloo(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        times, counts = res[rank]
        assert times == [float(world), 10.0 * world]
        assert counts == [float(sum(3 + r for r in range(world)))]
