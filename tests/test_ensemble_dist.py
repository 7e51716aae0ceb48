"""Sharding of ensemble instances over ranks (host logic, CPU gloo ranks):
greedy N log N balance and the final all-gather of per-instance metrics."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG


def test_partition_balances_and_covers():
    sys.path.insert(0, PKG)
    from ensemble import partition_instances
    rng = np.random.default_rng(0)
    sizes = np.round(np.exp(rng.uniform(np.log(2000), np.log(200000), 512))).astype(int)
    for world in (1, 2, 4, 8):
        parts = partition_instances(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        cost = [sum(sizes[i] * np.log(sizes[i]) for i in p) for p in parts]
        assert max(cost) / (sum(cost) / world) < 1.02


def _rank(rank, world, port, sizes, ret):
    sys.path.insert(0, PKG)
    import torch.distributed as dist
    from ensemble import gather_metrics, instance_metrics, partition_instances
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition_instances(sizes, world)[rank]
    rng = np.random.default_rng(1)
    # per-instance synthetic states (identical on every rank)
    from oracle import BODY_DTYPE
    states = []
    for n in sizes:
        b = np.zeros(n, BODY_DTYPE)
        b["mass"] = 1.0
        b["vx"] = rng.normal(size=n)
        b["vy"] = rng.normal(size=n)
        states.append(b)
    local = instance_metrics(np.concatenate([states[i] for i in mine]),
                             [sizes[i] for i in mine])
    full = gather_metrics(dist, mine, local, len(sizes))
    ref = instance_metrics(np.concatenate(states), sizes)
    ret[rank] = bool(np.allclose(full, ref, rtol=0, atol=0))
    dist.destroy_process_group()


def test_gather_metrics_two_ranks():
    sizes = [37, 400, 12, 999, 250, 3]
    mgr = mp.Manager()
    ret = mgr.dict()
    port = 29500 + os.getpid() % 1000
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, sizes, ret)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert ret[0] and ret[1]


def test_collective_device_follows_backend():
    sys.path.insert(0, PKG)
    import torch
    from ensemble import collective_device
    assert collective_device("gloo", 3) == torch.device("cpu")
    assert collective_device("nccl", 3) == torch.device("cuda", 3)
    assert collective_device("NCCL", 0) == torch.device("cuda", 0)


def _nccl_one_rank(port, ret):
    sys.path.insert(0, PKG)
    import datetime

    import torch
    import torch.distributed as dist
    from ensemble import gather_metrics
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    local = np.arange(12, dtype=np.float64).reshape(3, 4)
    full = gather_metrics(dist, [0, 2, 4], local, 5)
    ok = np.array_equal(full[[0, 2, 4]], local) and np.isnan(full[[1, 3]]).all()
    dist.destroy_process_group()
    ret["ok"] = bool(ok)


@pytest.mark.gpu
def test_gather_metrics_on_nccl():
    """The all-gather through NCCL itself (one rank on the one GPU; the
    buffers must be CUDA tensors there)."""
    mgr = mp.Manager()
    ret = mgr.dict()
    port = 28500 + os.getpid() % 1000
    p = mp.get_context("spawn").Process(target=_nccl_one_rank, args=(port, ret))
    p.start()
    p.join(180)
    assert p.exitcode == 0 and ret.get("ok")
