"""Generates ref_sigma_golden.npz: the reference's OWN depth-noise model (computeDepthMapStdevsPointwise
+ increaseStdevsNearDepthBoundaries, src/staticDepthNoiseModeling.cpp:85-137, 225-258, compiled in
place into oracle/_ref/libref_sigma.so by oracle/Makefile, with the L1 distance transform it takes
from OpenCV restated in oracle/ref_stubs_sigma) on seeded depth maps with holes and depth steps, the
inputs stored beside the outputs.  It pins the oracle's depth_sigma.

Run: python tests/golden/make_sigma_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "rgbd-flow_b200"))
import oracle_binding as ob  # noqa: E402
import synthetic as syn  # noqa: E402


def main():
    out = {}
    for tag, (W, H, seed) in {"a": (64, 48, 3), "b": (160, 120, 4), "c": (97, 61, 5)}.items():
        p = syn.make_pair(W=W, H=H, f=0.82 * W, cx=(W - 1) / 2, cy=(H - 1) / 2, n_patches=3, hole_frac=0.08, seed=seed)
        d = p["depth1"].astype(np.float32)
        out["in_" + tag] = d
        out["out_" + tag] = ob.depth_sigma(d, 4, impl="ref")
    np.savez_compressed(os.path.join(HERE, "ref_sigma_golden.npz"), **out)


if __name__ == "__main__":
    main()
