"""Rays across GPUs: one process per GPU, every rank holding a replica of the
scene (assets and triangles), each answering a contiguous share of the rays
with no collective on the data path. Rays are independent, so the shares
need no exchange; `gather_hits` is the one optional collective, an
all-gather of the hit records (over NCCL on GPUs, gloo on CPU) for callers
that want every answer on every rank. Serving spreads whole requests over
ranks instead (`request_owner`)."""
from __future__ import annotations

import numpy as np


def shard_range(n: int, rank: int, world: int):
    """[lo, hi) of rank's share of n rays: contiguous, sizes differing by at
    most one, in rank order, covering [0, n) exactly."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard")
    return rank * n // world, (rank + 1) * n // world


def request_owner(index: int, world: int) -> int:
    """The rank that serves request `index` of an arrival trace (round robin)."""
    return index % world


def gather_hits(local: np.ndarray, n_total: int, group=None) -> np.ndarray:
    """All-gather of each rank's hit records (any fixed-size numpy dtype,
    shares as shard_range cuts them) into the full array on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    size = local.dtype.itemsize
    share = max(shard_range(n_total, r, world)[1] - shard_range(n_total, r, world)[0] for r in range(world))
    buf = np.zeros(share * size, np.uint8)
    raw = np.ascontiguousarray(local).view(np.uint8).reshape(-1)
    buf[:raw.size] = raw
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.from_numpy(buf).to(dev)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    full = np.empty(n_total * size, np.uint8)
    for r, o in enumerate(outs):
        lo, hi = shard_range(n_total, r, world)
        full[lo * size:hi * size] = o.cpu().numpy()[:(hi - lo) * size]
    return full.view(local.dtype)
