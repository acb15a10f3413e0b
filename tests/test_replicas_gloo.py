"""Multi-process path of bench.py on CPU: two gloo ranks run the replica
aggregation (barrier, max-over-ranks time, whole-job throughput) exactly as
the NCCL ranks do on GPUs."""
from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import sys
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        ms = 2.0 + rank            # rank 1 is the slow one
        value, ms_max = bench.replica_value(1e9, ms, world)
        out[rank] = (value, ms_max)
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replica_aggregation():
    world = 2
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        value, ms_max = out[rank]
        assert ms_max == 3.0                       # max over ranks
        assert value == pytest.approx(2 * 1e9 / 3e-3 / 1e9)  # all ranks' work / slowest time


def test_passes_and_config():
    import sys
    sys.path.insert(0, str(ROOT))
    import bench
    assert [bench.passes_for(2 ** e, 32) for e in (4, 14, 15, 24)] == [1, 1, 2, 2]
    assert [bench.passes_for(2 ** e, 64) for e in (13, 14, 22)] == [1, 2, 2]
    assert bench.flops_per_transform(4096) == 5 * 4096 * 12
