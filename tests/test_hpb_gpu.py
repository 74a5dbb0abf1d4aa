"""HPB regularisation (the reference's default, -z 2) on the device against the oracle, on a B200.

The device restates the oracle's HPB step by step in the same float / double mix with every
operation rounded on its own, so most weights agree exactly.  Bit-for-bit agreement is not
promised: exp and the colour pyramid's FP32 values (from which the boundary heuristic takes an
8-bit colour, truncated) can differ in the last place.  Tolerances:
  * raw-depth pyramid (colour-guided fill + DepthMapPyramid): equal on >= 99.9 % of the pixels
  * regularisation weights per level (from the device's own colour pyramid and raw-depth levels):
    >= 99.5 % of the weights within 1e-6, mean |difference| <= 1e-3
  * the scene flow with HPB against the oracle's HPB solve: mean 3-D EPE <= 1 mm (the parity bar)
"""
import numpy as np
import pytest

import oracle_binding as ob
import rgbdflow as rf
import synthetic as syn

pytestmark = pytest.mark.gpu


def cam_of(p):
    c = p["cam"]
    return rf.CameraParams.make(p["W"], p["H"], c.f, c.cx, c.cy)


def hpb_params(W, n_outer=10):
    prm = rf.benchmark_params(W)
    prm.regularization = rf.REG_HPB
    prm.n_outer = n_outer
    return prm


@pytest.fixture(scope="module")
def solved(ctx):
    p = syn.make_config_pair("320x240", seed=5)
    prm = hpb_params(320, n_outer=1)
    cam = cam_of(p)
    flow, st = ctx.scene_flow_two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
    return p, prm, st


def test_hpb_raw_depth_pyramid_matches_oracle(ctx, solved):
    p, prm, st = solved
    col = p["bgr1"] / 255.0
    filled = ob.fill_small_regions_color(p["depth1"].astype(np.float64), col, 60)
    lev = ob.depth_map_pyramid(filled, prm.pyramid_ratio, prm.min_width)
    assert len(lev) == st.n_levels
    for k in range(st.n_levels):
        d = ctx.debug_plane(0, k, rf.PLANE_HPB_DEPTH)
        o = lev[k].astype(np.float32).astype(np.float64)
        same = np.mean(d == o)
        print("level %d: %.5f of the raw-depth pixels equal, max |diff| %.3g" % (k, same, np.abs(d - o).max()))
        assert same >= 0.999


def test_hpb_weights_match_oracle(ctx, solved):
    p, prm, st = solved
    for k in range(st.n_levels):
        img = np.stack([ctx.debug_plane(0, k, rf.PLANE_PYRAMID, c) for c in range(3)], -1)
        z = ctx.debug_plane(0, k, rf.PLANE_HPB_DEPTH)
        hpb = ob.heuristic_pb(img, z).astype(np.float64)
        H, W = z.shape
        for c in range(2):
            o = 1 - hpb[..., c] * .99
            if c == 0:
                o[:, W - 1] = 0
            else:
                o[H - 1, :] = 0
            d = ctx.debug_plane(0, k, rf.PLANE_REG, c)
            diff = np.abs(d - o.astype(np.float32))
            close = np.mean(diff <= 1e-6)
            print("level %d %s: %.5f within 1e-6, mean |diff| %.3g, max %.3g, weights in [%.3g, %.3g]"
                  % (k, "right" if c == 0 else "down", close, diff.mean(), diff.max(), d.min(), d.max()))
            assert close >= 0.995
            assert diff.mean() <= 1e-3
            inner = d[:, :W - 1] if c == 0 else d[:H - 1, :]  # the last column / row has no such neighbour (0)
            assert inner.min() >= 0.0099 and d.max() <= 1.0


@pytest.mark.parametrize("name", ["320x240", "640x480"])
def test_hpb_scene_flow_matches_oracle(ctx, name):
    p = syn.make_config_pair(name, seed=6)
    prm = hpb_params(p["W"])
    cam = cam_of(p)
    gpu, st = ctx.scene_flow_two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
    with ob.fill_order("rounds"):
        ref, rst = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
    mask = p["depth1"] > 0
    mean, mx = syn.epe3d(gpu, ref, p["z1_true"], p["cam"], mask)
    g = syn.epe3d(gpu, p["gt"], p["z1_true"], p["cam"], mask)[0]
    o = syn.epe3d(ref, p["gt"], p["z1_true"], p["cam"], mask)[0]
    print("%s HPB: EPE vs oracle mean %.3g mm max %.3g mm; vs ground truth device %.3g mm, oracle %.3g mm"
          % (name, mean * 1e3, mx * 1e3, g * 1e3, o * 1e3))
    assert np.isfinite(gpu).all()
    assert mean <= 1e-3


def test_hpb_warm_start_matches_oracle(ctx):
    """sceneFlowWithInit's HPB: the full-size colour with the raw (unfilled) depth."""
    p = syn.make_config_pair("320x240", seed=7)
    prm = hpb_params(320)
    cam = cam_of(p)
    est = (p["gt"] * 0.8).astype(np.float32)
    gpu, st = ctx.scene_flow_two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm, est_flow=est)
    with ob.fill_order("rounds"):
        ref, rst = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm, est_flow=est)
    mean, mx = syn.epe3d(gpu, ref, p["z1_true"], p["cam"], p["depth1"] > 0)
    print("HPB warm start: EPE vs oracle mean %.3g mm max %.3g mm" % (mean * 1e3, mx * 1e3))
    assert st.n_levels == 1
    assert mean <= 1e-3
