"""Generates tests/golden/ref_hpb_golden.npz from the reference's OWN DepthMapPyramid (the
raw-depth pyramid its HPB regularisation reads, src/depthMapPyramid.cpp), compiled from its
sources in place by oracle/Makefile (oracle/_ref/libref_hpb.so).  It pins the oracle's
depth_map_pyramid where the reference sources are absent.

Case (seeded; the input is stored beside the outputs): a 67x53 depth map, uniform in
[0.5, 4] m, a 0.5 m step at column 30, 20 % zero (invalid) pixels; ratios 0.75 (minWidth 20) and
0.5 (minWidth 10).

Run: python tests/golden/make_hpb_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle_binding as ob  # noqa: E402

CASES = {"r75": (0.75, 20), "r50": (0.5, 10)}


def depth_input():
    rng = np.random.default_rng(20261204)
    d = rng.uniform(0.5, 4.0, (53, 67))
    d[:, 30:] += 0.5
    d[rng.random(d.shape) < 0.2] = 0
    return d


if __name__ == "__main__":
    if not ob.ref_hpb_available():
        raise SystemExit("oracle/_ref/libref_hpb.so is not built (make -C oracle, with the reference present)")
    d = depth_input()
    out = {"depth": d}
    for tag, (ratio, mw) in CASES.items():
        levels = ob.depth_map_pyramid(d, ratio, mw, impl="ref")
        out[tag + "_n"] = np.array(len(levels))
        for i, lv in enumerate(levels):
            out["%s_%d" % (tag, i)] = lv
    dst = os.path.join(HERE, "ref_hpb_golden.npz")
    np.savez_compressed(dst, **out)
    print(dst, os.path.getsize(dst), "bytes")
