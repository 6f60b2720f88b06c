"""The C++ adapter header (include/dmap_b200.hpp) compiles against the C
ABI with a plain g++ (CPU), and, on a GPU, the single-ray intersect() and
intersect_batch() of a C++ caller give the Python binding's answers."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import dmap_b200 as dm
from dmap_b200 import scenes

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "adapter_quad.cpp"


def _build(tmp_path) -> Path:
    if not shutil.which("g++"):
        pytest.skip("g++ not found")
    exe = tmp_path / "adapter_quad"
    lib = dm.LIB_PATH
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           str(lib), f"-Wl,-rpath,{lib.parent}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_adapter_compiles_and_links(tmp_path):
    if not dm.LIB_PATH.exists():
        pytest.skip("library not built")
    assert _build(tmp_path).exists()


@pytest.mark.gpu
def test_adapter_answers_equal_python_binding(tmp_path):
    exe = _build(tmp_path)
    sc = scenes.quad_scene(64)
    nodes = sc.assets[0].nodes.astype(np.float32)
    rays = scenes.quad_camera_rays(24, 24).astype(np.float64)
    (tmp_path / "h.f32").write_bytes(nodes.tobytes())
    (tmp_path / "r.f64").write_bytes(rays.tobytes())
    r = subprocess.run([str(exe), str(nodes.shape[0]), str(tmp_path / "h.f32"), str(tmp_path / "r.f64"),
                        str(tmp_path / "o.f64")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = np.fromfile(tmp_path / "o.f64").reshape(-1, 12)
    ctx = dm.Context(0)
    dev = dm.Scene.from_synthetic(ctx, sc)
    h = dev.intersect(rays, dm.TraversalOptions(order="index", leaf_precision="f64"), np.float64)  # the adapter's flat-loop default
    hit = h["tri"] >= 0
    assert hit.sum() > 100
    assert np.array_equal(out[:, 1].astype(np.int32), h["tri"])
    assert np.array_equal(out[:, 11].astype(np.int32), h["tri"])
    assert np.array_equal(out[hit, 2], h["t"][hit]) and np.array_equal(out[hit, 10], h["t"][hit])
    assert np.array_equal(out[hit, 7:10], h["ng"][hit])
