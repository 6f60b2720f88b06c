"""The multi-GPU host logic on CPU: ray shares cover every ray once, and the
all-gather of hit records (gloo, world size 2 and 3, one process per rank)
rebuilds the single-process answer."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import dmap_b200 as dm
from dmap_b200.shard import gather_hits, request_owner, shard_range


@pytest.mark.parametrize("n", [0, 1, 7, 1000, 2_073_601])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shares_cover_every_ray_once(n, world):
    seen = np.zeros(n, np.int32)
    prev = 0
    for r in range(world):
        lo, hi = shard_range(n, r, world)
        assert lo == prev and hi - lo in (n // world, n // world + 1)
        seen[lo:hi] += 1
        prev = hi
    assert prev == n and (seen == 1).all()


def test_request_owner_round_robin():
    assert [request_owner(k, 4) for k in range(12)] == [0, 1, 2, 3] * 3


def _fake_hits(lo, hi):
    # a deterministic stand-in for each ray's answer
    h = np.zeros(hi - lo, dm.HIT32)
    k = np.arange(lo, hi)
    h["t"] = k * 0.5
    h["tri"] = np.where(k % 3 == 0, -1, k % 192)
    h["ng"] = np.stack([np.sin(k), np.cos(k), k % 5], 1)
    return h


def _rank(rank, world, port, n, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lo, hi = shard_range(n, rank, world)
        q.put((rank, gather_hits(_fake_hits(lo, hi), n).tobytes()))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,n", [(2, 1001), (3, 10)])
def test_gather_hits_gloo(world, n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = _fake_hits(0, n).tobytes()
    assert all(b == want for _, b in got)


_REC = np.dtype([("rec", "<f8", 12)])


def _scene_and_rays():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
    import py_oracle
    from dmap_b200 import scenes
    import helpers
    sc = helpers.small_sphere(16)
    cpu = py_oracle.CpuScene(py_oracle.Oracle(), sc)
    rays = np.concatenate([scenes.sphere_camera_rays(48, 27), helpers.near_surface_rays(cpu, 700)])
    return cpu, rays


def _query_rank(rank, world, port, q):
    """One rank of a replicated-scene query: the whole scene, its share of
    the rays answered through the CPU oracle, then the optional all-gather."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cpu, rays = _scene_and_rays()
        lo, hi = shard_range(len(rays), rank, world)
        h, _ = cpu.intersect(rays[lo:hi], order="nearest")
        local = np.ascontiguousarray(h).view(_REC).reshape(-1)
        q.put((rank, hi - lo, gather_hits(local, len(rays)).tobytes()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_query_equals_one_rank(world):
    """Each rank answers its share of real rays over its replica of the
    scene; the gathered answers equal one process answering them all."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_query_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    cpu, rays = _scene_and_rays()
    h, _ = cpu.intersect(rays, order="nearest")
    want = np.ascontiguousarray(h).view(_REC).reshape(-1).tobytes()
    assert sum(n for _, n, _ in got) == len(rays)
    assert all(b == want for _, _, b in got)
    assert (h[:, 10] >= 0).sum() > 100  # the shares hold real hits
