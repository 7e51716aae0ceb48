"""Batched ensemble: many independent simulations of uneven size advanced
together by one handle (every phase is one launch over all instances), and
the sharding of instances over GPUs.

Instances are independent, so a multi-GPU run partitions them over ranks
(greedy balance of sum N log N) with no exchange during the run; the only
collective is the final all-gather of per-instance metrics.
"""
from __future__ import annotations

import math

import numpy as np


def partition_instances(sizes, world: int):
    """Greedy longest-processing-time assignment by N log N.  Returns one
    sorted list of instance indices per rank."""
    cost = [n * math.log(max(n, 2)) for n in sizes]
    order = sorted(range(len(sizes)), key=lambda i: (-cost[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += cost[i]
    return [sorted(p) for p in parts]


def instance_metrics(bodies, sizes) -> np.ndarray:
    """Per instance: {kinetic energy, px, py, total mass} in float64."""
    out = np.zeros((len(sizes), 4))
    start = 0
    for k, n in enumerate(sizes):
        b = bodies[start:start + n]
        m = b["mass"].astype(np.float64)
        vx, vy = b["vx"].astype(np.float64), b["vy"].astype(np.float64)
        out[k] = (0.5 * np.sum(m * (vx * vx + vy * vy)), np.sum(m * vx),
                  np.sum(m * vy), np.sum(m))
        start += n
    return out


def collective_device(backend: str, local_rank: int):
    """Where a collective's buffers must live: NCCL moves only CUDA tensors
    (on the rank's own device), gloo only host tensors."""
    import torch
    if str(backend).lower() == "nccl":
        return torch.device("cuda", local_rank)
    return torch.device("cpu")


def gather_metrics(dist, local_ids, local_metrics, n_instances: int,
                   local_rank: int | None = None):
    """All-gather of per-instance metrics to every rank (the run's only
    collective).  `dist` is torch.distributed (gloo on CPU, nccl on GPU);
    the buffers are put where the group's backend needs them (for NCCL the
    rank's CUDA device: `local_rank`, default the current device)."""
    import torch
    world = dist.get_world_size()
    backend = dist.get_backend()
    if local_rank is None:
        local_rank = torch.cuda.current_device() if str(backend).lower() == "nccl" else 0
    dev = collective_device(backend, local_rank)
    host = torch.full((n_instances, local_metrics.shape[1] + 1), float("nan"),
                      dtype=torch.float64)
    for k, i in enumerate(local_ids):
        host[i, 0] = float(i)
        host[i, 1:] = torch.from_numpy(np.asarray(local_metrics[k], np.float64))
    buf = host.to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    full = torch.full_like(host, float("nan"))
    for p in parts:
        p = p.cpu()
        have = ~torch.isnan(p[:, 0])
        full[have] = p[have]
    return full[:, 1:].numpy()
