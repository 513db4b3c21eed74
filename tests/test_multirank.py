"""N > 1 path of bench.py on CPU: ranks solve independent systems and the job
time is the maximum over ranks (gloo, world_size 2, 127.0.0.1)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    local_ms = [100.0, 250.0][rank]
    out[rank] = bench.weak_throughput(local_ms, 30000 * 10, dist, "cpu")
    dist.destroy_process_group()


def test_weak_scaling_uses_max_over_ranks():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, value = out[r]
        assert ms == 250.0
        assert abs(value - 2 * 300000 / 0.25) < 1e-6


def test_single_rank_throughput():
    import bench
    ms, value = bench.weak_throughput(50.0, 1000)
    assert ms == 50.0 and value == 1000 / 0.05
