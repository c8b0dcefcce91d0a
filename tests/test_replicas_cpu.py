"""bench.py --gpus N runs N independent replicas of the workload (the path
has no exchange between GPUs): every rank times its own steps on the device
and the job's time is the max over ranks, with all ranks' cells counted. The
aggregation is checked here with two gloo ranks on the CPU."""
import os
import socket
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.replica_ms(10.0 * (rank + 1), world, "cpu")  # rank 1 is the slow replica
        value = bench.replica_value(1_000_000, 4, world, ms)
        (Path(out_dir) / ("r%d" % rank)).write_text("%r %r" % (ms, value))
    finally:
        dist.destroy_process_group()


def test_replica_time_is_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.spawn(_rank, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        ms, value = (float(v) for v in (tmp_path / ("r%d" % r)).read_text().split())
        assert ms == 20.0
        assert value == pytest.approx(1_000_000 * 4 * world / 0.020 / 1e6)


def test_single_rank_passthrough():
    sys.path.insert(0, str(REPO))
    import bench

    assert bench.replica_ms(12.5, 1, "cpu") == 12.5
    assert bench.replica_value(2_000_000, 10, 1, 1000.0) == pytest.approx(20.0)
