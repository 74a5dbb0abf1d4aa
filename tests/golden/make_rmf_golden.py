"""Generates ref_rmf_golden.npz: the reference's OWN recursive median hole fill
(recursiveMedianFilterAux, src/recursiveMedianFiltering.cpp:35-99, compiled in place into
oracle/_ref/libref_rmf.so by oracle/Makefile) on seeded depth maps with clustered holes, the
inputs stored beside the outputs.  It pins the oracle's median_fill, whose fill order (the
libstdc++ hash-set order) the reference's result depends on.

Run: python tests/golden/make_rmf_golden.py
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
    for tag, (W, H, frac, seed) in {"a": (64, 48, 0.08, 3), "b": (160, 120, 0.08, 4), "c": (97, 61, 0.15, 5)}.items():
        p = syn.make_pair(W=W, H=H, f=0.82 * W, cx=(W - 1) / 2, cy=(H - 1) / 2, n_patches=2, hole_frac=frac, seed=seed)
        d = p["depth1"].astype(np.float64)
        out["in_" + tag] = d
        out["out_" + tag] = ob.median_fill(d, impl="ref")
    np.savez_compressed(os.path.join(HERE, "ref_rmf_golden.npz"), **out)


if __name__ == "__main__":
    main()
