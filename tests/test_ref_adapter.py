"""The drop-in adapter over the reference's own types
(include/dmap_b200_reference.hpp: dmap::GpuObjectIntersector, constructed
from std::vector<BaseTriangle>, TaylorPyramid and HeightGrid, with
ObjectIntersector::intersect's signature, displaced_intersector.h:183-197).

On the CPU the adapter and its check driver (tests/cpp/ref_adapter_check.cpp)
compile against the reference's headers in the checkout, with the oracle's
stand-ins for its missing submodules. On the GPU the driver, built by
`make -C oracle ref_adapter` beside the reference sources, builds the
reference's ObjectIntersector and the adapter from the same BaseTriangles and
answers every ray through both: hits, triangles and texels must be equal bit
for bit, through the single-ray call and the batch call alike."""
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
REF_SRC = Path(os.environ.get("DMAP_REF_ROOT", "/root/reference")) / "code" / "cpp" / "src"
CHECK = ROOT / "oracle" / "_ref" / "ref_adapter_check"


@pytest.mark.skipif(not (REF_SRC / "displaced_intersector.h").exists(), reason="reference checkout not present")
def test_adapter_compiles_against_the_reference_headers():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-w", f"-I{ROOT / 'oracle' / 'ref_shim'}",
                        f"-I{REF_SRC}", f"-I{ROOT / 'include'}", str(ROOT / "tests" / "cpp" / "ref_adapter_check.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def _write_input(path, nodes, scale, offset, repeat, tris, rays, build=0):
    with open(path, "wb") as f:
        np.array([nodes.shape[0], build, int(repeat)], np.int32).tofile(f)
        np.array([scale, offset], np.float64).tofile(f)
        np.ascontiguousarray(nodes, np.float64).tofile(f)
        np.array([len(tris)], np.int32).tofile(f)
        np.ascontiguousarray(tris, np.float64).tofile(f)
        np.array([len(rays)], np.int32).tofile(f)
        np.ascontiguousarray(rays, np.float64).tofile(f)


def _cases():
    import helpers
    from dmap_b200 import scenes
    quad = scenes.quad_scene(64)
    charts = helpers.chart_scene(32)
    return [("quad", quad, 0), ("charts", charts, 0), ("quad-direct", quad, 1)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 2], ids=["quad", "charts", "quad-direct"])
def test_adapter_equals_object_intersector(oracle, case):
    if not CHECK.exists():
        pytest.skip("oracle/_ref/ref_adapter_check not built (make -C oracle ref_adapter)")
    import py_oracle
    import helpers
    from dmap_b200 import scenes
    name, sc, build = _cases()[case]
    # one object: the scene's first asset and the triangles it displaces
    a = sc.assets[0]
    tris = sc.tris[sc.tri_asset == 0]
    sub = scenes.Scene([a], tris, np.zeros(len(tris), np.int32))
    cpu = py_oracle.CpuScene(oracle, sub)
    rays = np.concatenate([helpers.near_surface_rays(cpu, 600), helpers.aimed_rays(cpu, 600)[0]]).astype(np.float64)
    if name.startswith("quad"):
        rays = np.concatenate([rays, scenes.quad_camera_rays(24, 24).astype(np.float64)])
    with tempfile.TemporaryDirectory() as d:
        fin, fout = Path(d) / "in.bin", Path(d) / "out.bin"
        _write_input(fin, a.nodes, a.scale, a.offset, a.repeat, tris, rays, build)
        r = subprocess.run([str(CHECK), str(fin), str(fout)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        out = np.fromfile(fout, np.float64).reshape(len(rays), 48)
    ref, one, batch = out[:, 0:12], out[:, 12:24], out[:, 24:36]
    s_ref, s_one = out[:, 36:42], out[:, 42:48]
    hit = ref[:, 10] >= 0
    assert hit.sum() > len(rays) // 4
    # the adapter's answers are the reference's, bit for bit
    assert np.array_equal(one.tobytes(), ref.tobytes())
    assert np.array_equal(batch.tobytes(), ref.tobytes())
    # the counters are the device walk's own: a hit took a leaf test there too
    assert (s_one[hit, 2] >= 1).all() and (s_ref[hit, 2] >= 1).all()
