"""The oracle's pyramid against the reference's golden vectors and the
reference's own pyramid tests (code/python/poc/tests/test_pyramid.py,
code/cpp/src/validate_pyramid.cpp)."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"
CHANNELS = ("h0", "gu", "gv", "r", "ru", "rv", "h_min", "h_max")
CASES = ["random_65", "random_33", "step_17", "ramp_17"]


def load(case):
    z = np.load(GOLDEN / f"pyramid_{case}.npz")
    return z["values"], float(z["scale"][0]), z


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("build", ["fold", "direct"])
def test_oracle_matches_golden(oracle, case, build):
    """validate_pyramid.cpp:111-164 demands a scaled error <= 1e-12; the
    restatement follows the numpy arithmetic step for step, so it is exact."""
    values, scale, z = load(case)
    levels = oracle.pyramid(values, scale, 0.0, build)
    assert len(levels) == sum(1 for k in z.files if k.startswith(f"{build}/h0_L"))
    for k, lv in enumerate(levels):
        for ch in CHANNELS:
            g = z[f"{build}/{ch}_L{k}"]
            mag = max(np.abs(g).max(), 1.0)
            assert np.abs(lv[ch] - g).max() <= 1e-12 * mag, (case, build, k, ch)
            assert np.array_equal(lv[ch], g), (case, build, k, ch)


def _bilinear(values, scale, X, Y):
    n = values.shape[0] - 1
    fx, fy = X * n, Y * n
    i = np.minimum(fx.astype(np.int64), n - 1)
    j = np.minimum(fy.astype(np.int64), n - 1)
    s, t = fx - i, fy - j
    v = values * scale
    h = ((1 - s) * (1 - t) * v[j, i] + s * (1 - t) * v[j, i + 1] + (1 - s) * t * v[j + 1, i]
         + s * t * v[j + 1, i + 1])
    hu = ((1 - t) * (v[j, i + 1] - v[j, i]) + t * (v[j + 1, i + 1] - v[j + 1, i])) * n
    hv = ((1 - s) * (v[j + 1, i] - v[j, i]) + s * (v[j + 1, i + 1] - v[j, i + 1])) * n
    return h, hu, hv


@pytest.mark.parametrize("case", ["random_33", "step_17"])
@pytest.mark.parametrize("build", ["fold", "direct"])
def test_containment(oracle, case, build):
    """test_pyramid.py:34-51: dense samples lie in every ancestor's slab,
    gradient intervals and height range (5 samples per texel axis)."""
    values, scale, _ = load(case)
    levels = oracle.pyramid(values, scale, 0.0, build)
    n = values.shape[0] - 1
    x = (np.arange(n * 5) + 0.5) / (n * 5)
    X, Y = np.meshgrid(x, x, indexing="xy")
    h, hu, hv = _bilinear(values, scale, X, Y)
    tol = 1e-10
    for level, lv in enumerate(levels):
        w = 2.0 ** level / n
        m = lv["h0"].shape[0]
        ci = np.minimum((X / w).astype(np.int64), m - 1)
        cj = np.minimum((Y / w).astype(np.int64), m - 1)
        u0, v0 = (ci + 0.5) * w, (cj + 0.5) * w
        plane = lv["h0"][cj, ci] + lv["gu"][cj, ci] * (X - u0) + lv["gv"][cj, ci] * (Y - v0)
        assert (np.abs(h - plane) <= lv["r"][cj, ci] + tol).all()
        assert (np.abs(hu - lv["gu"][cj, ci]) <= lv["ru"][cj, ci] + tol).all()
        assert (np.abs(hv - lv["gv"][cj, ci]) <= lv["rv"][cj, ci] + tol).all()
        assert (h >= lv["h_min"][cj, ci] - tol).all() and (h <= lv["h_max"][cj, ci] + tol).all()


def test_offset_shifts_value_channels_only(oracle):
    """taylor_pyramid.cpp:239-250: a constant offset moves h0, h_min and h_max."""
    values, scale, _ = load("random_33")
    a = oracle.pyramid(values, scale, 0.0)
    b = oracle.pyramid(values, scale, 0.25)
    for la, lb in zip(a, b):
        for ch in ("gu", "gv", "r", "ru", "rv"):
            assert np.array_equal(la[ch], lb[ch])
        for ch in ("h0", "h_min", "h_max"):
            assert np.array_equal(la[ch] + 0.25, lb[ch])


def test_bad_grid_rejected(oracle):
    with pytest.raises(ValueError):
        oracle.pyramid(np.zeros((10, 10)))


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("build", ["fold", "direct"])
def test_reference_build_matches_golden(reference, case, build):
    """The reference's C++ TaylorPyramid, compiled here, against its numpy
    golden vectors: the pin of the pin."""
    values, scale, z = load(case)
    for k, lv in enumerate(reference.pyramid(values, scale, 0.0, build)):
        for ch in CHANNELS:
            assert np.array_equal(lv[ch], z[f"{build}/{ch}_L{k}"]), (case, build, k, ch)
