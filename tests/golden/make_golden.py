"""Regenerates the golden pyramid fixtures from the reference's own numpy
pyramid (code/python/poc/dmapref/pyramid.py in MangoSister/dmap).

The reference exports its golden pyramids with
experiments/export_golden_pyramid.py; of its three cases only random_65
(seed 2027, scale 1.0) can be regenerated, because the two texture cases
need image assets that are not in the checkout. This script writes that case
and three small known-answer maps from the reference's tests
(tests/test_pyramid.py): a 33^2 random map at scale 0.4, the 17^2 step edge
and the 17^2 ramp. Both build modes, every level, all eight channels.

Run in a checkout that holds the reference; its root is the first argument,
else $DMAP_REF_ROOT, else /root/reference:
python tests/golden/make_golden.py [REF_ROOT]
"""
import sys
from pathlib import Path

import numpy as np

import os

REF = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DMAP_REF_ROOT", "/root/reference"))
sys.path.insert(0, str(REF / "code" / "python" / "poc"))
from dmapref.pyramid import BUILDS, CHANNELS, TaylorPyramid  # noqa: E402

OUT = Path(__file__).resolve().parent


def export(name, values, scale):
    arrays = {"values": np.asarray(values, np.float64), "scale": np.array([scale])}
    for build in BUILDS:
        pyr = TaylorPyramid(values, scale, build)
        for k, level in enumerate(pyr.levels):
            for ch in CHANNELS:
                arrays[f"{build}/{ch}_L{k}"] = level[ch]
    np.savez_compressed(OUT / f"pyramid_{name}.npz", **arrays)


def main():
    rng = np.random.default_rng(2027)
    export("random_65", rng.random((65, 65)), 1.0)       # export_golden_pyramid.py:48
    rng = np.random.default_rng(11)
    export("random_33", rng.random((33, 33)), 0.4)       # test_pyramid.py:82,99
    step = np.zeros((17, 17))
    step[:, 9:] = 1.0
    export("step_17", step, 1.0)                          # test_pyramid.py:88-90
    jj, ii = np.mgrid[0:17, 0:17]
    export("ramp_17", 0.3 * ii / 16 - 0.2 * jj / 16, 1.0)  # test_pyramid.py:141-142


if __name__ == "__main__":
    main()
