"""Generates the golden fixtures in this directory from the reference's OWN code, compiled from
its sources in place by oracle/Makefile (oracle/_ref).  The reference ships no tests or golden
data, so these fixtures are how the CPU restatement (oracle/) is pinned.

  python tests/golden/make_golden.py           CPU part: ref_cpu_golden.npz
                                                (GaussianPyramid, Image::imresize, im2feature
                                                 sequence, ImageProcessing::warpImage)
  python tests/golden/make_golden.py --cuda    GPU part: ref_cuda_golden.npz (sceneFlowSingleScale,
                                                the reference's CUDA solver, on a B200)
Inputs are seeded; the inputs are stored beside the outputs.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "rgbd-flow_b200"))
import oracle_binding as ob  # noqa: E402


def cpu_cases():
    rng = np.random.default_rng(20240601)
    out = {}
    for tag, (W, H) in {"a": (37, 29), "b": (44, 34)}.items():
        img = rng.random((H, W, 3))
        out["img_" + tag] = img
        for rtag, (ratio, mw) in {"r50": (0.5, 4), "r75": (0.75, 20)}.items():
            levels = ob.build_pyramid(img, ratio, mw, impl="ref")
            out["pyr_%s_%s_n" % (tag, rtag)] = np.array(len(levels))
            for i, lv in enumerate(levels):
                out["pyr_%s_%s_%d" % (tag, rtag, i)] = lv
        feat = ob.im2feature(img, impl="ref")
        out["feat_" + tag] = feat
        out["up_" + tag] = ob.resize_dims(img[:, :, 1], 2 * W + 1, 2 * H - 1, impl="ref")
        f2 = rng.random((H, W, 5))
        d1 = rng.uniform(0.5, 3, (H, W))
        d2 = rng.uniform(0.5, 3, (H, W))
        u = rng.normal(0, 3, (H, W))
        v = rng.normal(0, 3, (H, W))
        w = rng.normal(0, 0.05, (H, W))
        wi, wd = ob.warp(feat, d1, f2, d2, u, v, w, impl="ref")
        for k, x in dict(f2=f2, d1=d1, d2=d2, u=u, v=v, w=w, wi=wi, wd=wd).items():
            out["warp_%s_%s" % (tag, k)] = x
    return out


def cuda_cases():
    """Single-level inputs built by the oracle from a seeded synthetic pair, solved by the
    reference's CUDA sceneFlowSingleScale."""
    import rgbdflow as rf
    import synthetic as syn
    out = {}
    for tag, (W, H, early) in {"s": (48, 36, 0), "e": (64, 48, 1)}.items():
        p = syn.make_pair(W=W, H=H, f=W * 0.82, cx=(W - 1) / 2, cy=(H - 1) / 2, n_patches=2, hole_frac=0.0,
                          seed=11 if tag == "s" else 12)
        im1 = p["bgr1"] / 255.0
        im2 = p["bgr2"] / 255.0
        f1 = ob.im2feature(im1)
        f2 = ob.im2feature(im2)
        d1 = p["depth1"].astype(np.float64)
        d2 = p["depth2"].astype(np.float64)
        sig = ob.depth_sigma(p["depth1"])
        ddw = ob.stereo_error1() / sig.astype(np.float64)
        dsw = np.full((H, W), float(np.float32(W * 0.82)) ** 2)
        mag = (float(np.float32(W * 0.82)) / d1) ** 2
        regw = np.ones((H, W, 2))
        regw[:, -1, 0] = 0
        regw[-1, :, 1] = 0
        u0 = np.full((H, W), 0.3)
        v0 = np.full((H, W), -0.2)
        w0 = np.zeros((H, W))
        wi, wd = ob.warp(f1, d1, f2, d2, u0, v0, w0)
        args = dict(f1=f1, d1=d1, f2=f2, d2=d2, wi=wi, wd=wd, u=u0, v=v0, w=w0, ddw=ddw, dsw=dsw, mag=mag, regw=regw)
        fl = np.float32(W * 0.82)
        res = ob.single_scale(float(fl), f1, d1, f2, d2, wi, wd, u0, v0, w0, 1.0, ddw, 0.02, dsw, 1e-5, mag, regw,
                              4, 1, 30, early, impl="ref")
        for k, x in args.items():
            out["%s_%s" % (tag, k)] = x
        out["%s_f" % tag] = np.array(fl)
        out["%s_early" % tag] = np.array(early)
        out["%s_out_u" % tag], out["%s_out_v" % tag], out["%s_out_w" % tag] = res[0], res[1], res[2]
    return out


if __name__ == "__main__":
    if "--cuda" in sys.argv:
        dst = sys.argv[sys.argv.index("--out") + 1] if "--out" in sys.argv else os.path.join(HERE, "ref_cuda_golden.npz")
        np.savez_compressed(dst, **cuda_cases())
    else:
        np.savez_compressed(os.path.join(HERE, "ref_cpu_golden.npz"), **cpu_cases())
    print("ok")
