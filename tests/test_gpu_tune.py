"""The schedule autotuner: it returns one of its candidate launch shapes,
remembers it in the cache file, and the tuned schedule answers exactly like
the default one."""
import numpy as np
import pytest

import dmap_b200 as dm
import py_oracle
import helpers
from dmap_b200 import scenes

pytestmark = pytest.mark.gpu


def test_autotune_picks_a_candidate_and_caches_it(oracle, tmp_path):
    torch = pytest.importorskip("torch")
    ctx = dm.Context(0)
    sc = helpers.small_sphere(32)
    cpu = py_oracle.CpuScene(oracle, sc)
    dev = dm.Scene.from_synthetic(ctx, sc)
    rays = np.concatenate([scenes.sphere_camera_rays(128, 72), helpers.near_surface_rays(cpu, 4000)])
    rd = torch.from_numpy(rays).cuda()
    cache = tmp_path / "tune.txt"
    best, ms = dev.autotune(rd.data_ptr(), dm.F32, len(rays), cache_path=str(cache))
    assert best.rounds in (2, 3, 4, 6, 8, 12) and best.blocks_per_sm in (3, 4, 5) and ms > 0
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and lines[0].split()[1:3] == [str(best.rounds), str(best.blocks_per_sm)]
    again, ms2 = dev.autotune(rd.data_ptr(), dm.F32, len(rays), cache_path=str(cache))
    assert (again.rounds, again.blocks_per_sm) == (best.rounds, best.blocks_per_sm) and ms2 == pytest.approx(ms)
    assert len(cache.read_text().splitlines()) == 1
    a = dev.intersect(rays, best, np.float64)
    b = dev.intersect(rays, dm.TraversalOptions(), np.float64)
    assert a.tobytes() == b.tobytes()
