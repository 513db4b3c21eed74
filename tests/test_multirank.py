"""N > 1 paths on CPU (gloo, world_size 2, 127.0.0.1).

* bench.py: ranks solve independent systems and the job time is the maximum
  over ranks.
* Node-range sharding (`glst_create_shard`): the reference splits the
  cubature nodes into contiguous per-GPU ranges and sums the per-atom
  outputs with an NCCL reduce (src/glst_force.cu:276-293, :1584-1602,
  src/device_comm.cu:176-201).  Here each rank evaluates its node range with
  the FP64 oracle (rank 0 also the near field) and the ranks sum the four
  per-atom rows with a gloo all-reduce; the sum must be the unsharded solve
  and match the reference's own outputs.
"""
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
    mgr = mp.get_context("spawn").Manager()  # no fork of a threaded test process
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


def _shard_rank(rank, world, port, case, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import numpy as np
    import __graft_entry__
    from oracle import oracle, planner
    from test_golden import load_case
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    g = __graft_entry__.load_package()
    d, (x, y, z, q), box = load_case(case, "double")
    p = planner.make_plan(len(x), float(d["tol"]), box, float(d["rcut"]), planner.TDesignStore(g.TDESIGN_STORE))
    k0, k1 = p.K * rank // world, p.K * (rank + 1) // world
    part = oracle.glst(x, y, z, q, p, k0=k0, k1=k1, far=True, sr=(rank == 0))
    t = torch.from_numpy(np.stack(part))
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out[rank] = (t.numpy().copy(), k0, k1, p.K)
    dist.destroy_process_group()


@pytest.mark.parametrize("case", ["w1000_tol1e-4"])
def test_node_shards_sum_over_gloo(store, case):
    import numpy as np
    from oracle import oracle, planner
    from test_golden import load_case
    world = 2
    mgr = mp.get_context("spawn").Manager()  # no fork of a threaded test process
    out = mgr.dict()
    mp.spawn(_shard_rank, args=(world, _free_port(), case, out), nprocs=world, join=True)
    d, (x, y, z, q), box = load_case(case, "double")
    p = planner.make_plan(len(x), float(d["tol"]), box, float(d["rcut"]), store)
    full = np.stack(oracle.glst(x, y, z, q, p))
    ranges = sorted((out[r][1], out[r][2]) for r in range(world))
    assert ranges[0][0] == 0 and ranges[-1][1] == p.K and ranges[0][1] == ranges[1][0]
    for r in range(world):
        summed = out[r][0]
        assert np.array_equal(summed, out[0][0])  # every rank holds the same sum
        scale = np.abs(full).max(axis=1, keepdims=True)
        assert np.all(np.abs(summed - full) <= 1e-12 * scale), np.abs(summed - full).max()
    rep = oracle.error_report(tuple(out[0][0]), (d["fx"], d["fy"], d["fz"], d["en"]))
    assert rep["force_rms_rel"] <= 1e-12 and rep["energy_rel"] <= 1e-12, rep
