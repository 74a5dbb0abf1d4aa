"""Generates tests/golden/ref_flow2d_golden.npz from the reference's OWN 2-D optical-flow code
(OpticalFlow::Coarse2FineFlow with SmoothFlowSOR, the demo's flow type 1), compiled from its
sources in place by oracle/Makefile (oracle/_ref/libref_flow2d.so).  It pins the oracle's 2-D
restatement where the reference sources are absent.

Cases (seeded; the inputs are stored beside the outputs):
  shift: a smooth random texture, 72x56, moved by (1.5, 0.5) px; the demo's parameters
         (alpha 0.02, ratio 0.75, minWidth 20, 10 outer, 1 inner, 400 SOR iterations)
  patch: two frames of a textured-patch scene at 96x72 (rgbd-flow_b200/synthetic.py), alpha
         0.05, ratio 0.5, minWidth 12, 7 outer, 2 inner, 30 SOR iterations

Run: python tests/golden/make_flow2d_golden.py
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

PARAMS = {
    "shift": dict(alpha=0.02, ratio=0.75, min_width=20, n_outer=10, n_inner=1, n_sor=400),
    "patch": dict(alpha=0.05, ratio=0.5, min_width=12, n_outer=7, n_inner=2, n_sor=30),
}


def smooth_texture(rng, H, W, pad=8):
    """A random colour texture smoothed with a 5x5 box filter twice, in [0, 255]."""
    t = rng.random((H + 2 * pad, W + 2 * pad, 3))
    for _ in range(2):
        acc = np.zeros_like(t)
        for dy in range(-2, 3):
            for dx in range(-2, 3):
                acc += np.roll(np.roll(t, dy, 0), dx, 1)
        t = acc / 25
    t = (t - t.min()) / (t.max() - t.min())
    return t * 255.0


def bilinear_shift(img, dx, dy):
    """img sampled at (x - dx, y - dy): content moved by (+dx, +dy)."""
    H, W = img.shape[:2]
    y, x = np.mgrid[0:H, 0:W].astype(np.float64)
    xs, ys = np.clip(x - dx, 0, W - 1), np.clip(y - dy, 0, H - 1)
    x0, y0 = np.floor(xs).astype(int), np.floor(ys).astype(int)
    x1, y1 = np.minimum(x0 + 1, W - 1), np.minimum(y0 + 1, H - 1)
    fx, fy = (xs - x0)[..., None], (ys - y0)[..., None]
    return ((1 - fx) * (1 - fy) * img[y0, x0] + fx * (1 - fy) * img[y0, x1] + (1 - fx) * fy * img[y1, x0]
            + fx * fy * img[y1, x1])


def cases():
    rng = np.random.default_rng(20261203)
    H, W, pad = 56, 72, 8
    tex = smooth_texture(rng, H, W, pad)
    moved = bilinear_shift(tex, 1.5, 0.5)
    shift1 = np.rint(tex[pad:pad + H, pad:pad + W]).astype(np.uint8)
    shift2 = np.rint(moved[pad:pad + H, pad:pad + W]).astype(np.uint8)
    p = syn.make_pair(W=96, H=72, f=78.75, cx=47.5, cy=35.5, n_patches=3, hole_frac=0.0, seed=77)
    out = {}
    for tag, (b1, b2) in {"shift": (shift1, shift2), "patch": (p["bgr1"], p["bgr2"])}.items():
        u, v = ob.optical_flow_2d(b1, b2, impl="ref", **PARAMS[tag])
        out[tag + "_bgr1"], out[tag + "_bgr2"] = np.ascontiguousarray(b1), np.ascontiguousarray(b2)
        out[tag + "_u"], out[tag + "_v"] = u, v
    return out


if __name__ == "__main__":
    if not ob.ref_flow2d_available():
        raise SystemExit("oracle/_ref/libref_flow2d.so is not built (make -C oracle, with the reference present)")
    dst = os.path.join(HERE, "ref_flow2d_golden.npz")
    np.savez_compressed(dst, **cases())
    print(dst, os.path.getsize(dst), "bytes")
