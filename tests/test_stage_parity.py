"""Per-stage parity of the sm_100a solve with the CPU oracle, on a B200.

Each test runs the library through its C ABI, reads a stage's device planes back
(rgbdflow_debug_read_plane) and recomputes that stage on the CPU from the device's own inputs to the
stage, so every stage is checked on its own and an error cannot hide behind the SOR's damping.

Tolerances ("rel" = largest |device - oracle| over a plane, divided by the plane's largest |oracle|):
  * pyramid levels (GaussianPyramid: Gaussian filter + bilinear resize) from the device's level-0
    planes:                                     rel <= 2e-6 (FP32 accumulation of <= 13-tap sums)
  * level inputs (im2feature, depth-magnitude and regularisation weights) from the device's
    pyramid planes:                             rel <= 2e-6 (LETOUZEY's exp: rel <= 1e-5)
  * hole fill: the device's filled depths equal the oracle's restatement of the device's fill
    order (parallel rounds) bit for bit
  * depth sigma (through the level-0 depth-data weight): within one float rounding
  * one linearisation (the compact 12-coefficient system against the reference's 8 planes): per
    coefficient plane, rel <= 10 x (the oracle's own change when its inputs are rounded to FP32,
    as the device stores them) + 1e-5.  The robust depth weight pi = 1 / (2 sqrt(e^2 + 1e-10))
    makes the data-term coefficients sensitive to the last bit of the inputs (the FP32 rounding
    alone moves them by up to ~1e-3), while the regularisation coefficients stay within ~3e-7.
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


def rel(dev, ora):
    scale = np.abs(ora).max()
    return float(np.abs(dev - ora).max() / scale) if scale > 0 else float(np.abs(dev).max())


def solve(ctx, p, prm):
    cam = cam_of(p)
    return ctx.scene_flow_two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)


@pytest.fixture(scope="module")
def solved(ctx):
    p = syn.make_config_pair("320x240", seed=1)
    prm = rf.benchmark_params(320)
    flow, st = solve(ctx, p, prm)
    return p, prm, flow, st


def test_pyramid_levels_match_oracle(ctx, solved):
    p, prm, _, st = solved
    worst = 0.0
    for z in range(10):
        base = ctx.debug_plane(0, 0, rf.PLANE_PYRAMID, z)
        lev = ob.build_pyramid(base, prm.pyramid_ratio, prm.min_width)
        assert len(lev) == st.n_levels
        for k in range(1, st.n_levels):
            d = ctx.debug_plane(0, k, rf.PLANE_PYRAMID, z)
            assert d.shape == lev[k].shape
            r = rel(d, lev[k])
            worst = max(worst, r)
            assert r <= 2e-6, "plane %d level %d: rel %.3g" % (z, k, r)
    print("pyramids: worst rel %.3g" % worst)


def test_level_inputs_match_oracle(ctx, solved):
    p, prm, _, st = solved
    cam_full = cam_of(p)
    worst = {}
    for k in range(st.n_levels):
        pyr = [ctx.debug_plane(0, k, rf.PLANE_PYRAMID, z) for z in range(10)]
        for f, kind in ((0, rf.PLANE_FEATURES1), (1, rf.PLANE_FEATURES2)):
            feat = ob.im2feature(np.stack(pyr[3 * f:3 * f + 3], -1))
            for c in range(5):
                r = rel(ctx.debug_plane(0, k, kind, c), feat[..., c])
                worst["features"] = max(worst.get("features", 0), r)
                assert r <= 2e-6, "level %d frame %d channel %d: rel %.3g" % (k, f, c, r)
        for f in range(2):
            # the linearisation reads the pyramid's depth planes unchanged (FP32 storage)
            assert np.array_equal(ctx.debug_plane(0, k, rf.PLANE_DEPTH, f), pyr[6 + f])
        r = rel(ctx.debug_plane(0, k, rf.PLANE_DEPTH_MAG, 0), ob.depth_mag_weights(pyr[6], cam_full))
        worst["depth_mag"] = max(worst.get("depth_mag", 0), r)
        assert r <= 2e-6, "level %d depth-magnitude weight: rel %.3g" % (k, r)
        reg = ob.reg_weights(pyr[6], rf.REG_ISOTROPIC)
        for c in range(2):
            assert np.array_equal(ctx.debug_plane(0, k, rf.PLANE_REG, c), reg[..., c])
    print("level inputs: worst rel %s" % worst)


def test_depth_sigma_weights_match_oracle(ctx, solved):
    """The device's depth sigma (k_sigma: the boundary distance by an exact L1 search) through the
    level-0 depth-data weight stereoError(1) / sigma, against the oracle's sigma (itself equal to
    the reference's own depth-noise model): within one float rounding (the boundary increase goes
    through exp and log, whose last bit CUDA and the C library may round differently)."""
    p, prm, _, _ = solved
    sig = ob.depth_sigma(p["depth1"], 4).astype(np.float64)
    expect = (ob.stereo_error1() / sig * prm.depth_vs_color_data_weight).astype(np.float32).astype(np.float64)
    dev = ctx.debug_plane(0, 0, rf.PLANE_PYRAMID, 8)
    r = np.abs(dev - expect) / np.abs(expect)
    print("depth-data weights: %.5f equal, max rel %.3g" % (np.mean(dev == expect), r.max()))
    assert r.max() <= 2.4e-7


def test_letouzey_weights_match_oracle(ctx):
    p = syn.make_config_pair("320x240", seed=2)
    prm = rf.benchmark_params(320)
    prm.regularization = rf.REG_LETOUZEY
    prm.n_outer = 1
    _, st = solve(ctx, p, prm)
    worst = 0.0
    for k in range(st.n_levels):
        reg = ob.reg_weights(ctx.debug_plane(0, k, rf.PLANE_PYRAMID, 6), rf.REG_LETOUZEY)
        for c in range(2):
            r = rel(ctx.debug_plane(0, k, rf.PLANE_REG, c), reg[..., c])
            worst = max(worst, r)
            assert r <= 1e-5, "level %d channel %d: rel %.3g" % (k, c, r)
    print("LETOUZEY weights: worst rel %.3g" % worst)


@pytest.mark.parametrize("name", ["320x240", "640x480"])
def test_filled_depth_equals_rounds_fill(ctx, name):
    """The device's hole fill against the oracle's restatement of its order, on the configurations'
    clustered holes: every filled value equal."""
    p = syn.make_config_pair(name, seed=4)
    prm = rf.benchmark_params(p["W"])
    solve(ctx, p, prm)
    for f, key in enumerate(("depth1", "depth2")):
        ref, rounds = ob.median_fill_rounds(p[key])
        dev = ctx.debug_plane(0, 0, rf.PLANE_PYRAMID, 6 + f)
        hole = p[key] <= 0
        assert hole.sum() > 0
        assert np.array_equal(dev, ref.astype(np.float32).astype(np.float64)), "frame %d" % (f + 1)
        st = ctx.debug_plane(0, 0, rf.PLANE_FILL_ROUND, f)
        assert np.all(st[~hole] == 0) and np.all((st[hole] >= 1) & (st[hole] <= rounds))
        assert st[hole].max() == rounds
        print("%s frame %d: %d holes filled in %d rounds" % (name, f + 1, hole.sum(), rounds))


def test_hole_pixel_flow_against_reference_fill(ctx):
    """Where the fill order matters: the flow on frame-1 hole pixels (3-D EPE with the true depth),
    the device against the oracle with the reference's fill order, and both against ground truth.
    The device's parallel fill may give a hole pixel another median than the reference's hash-set
    order; its flow there must be as accurate as the reference's."""
    p = syn.make_config_pair("640x480", seed=0)
    prm = rf.benchmark_params(640)
    gpu, _ = solve(ctx, p, prm)
    cam = cam_of(p)
    ref, _ = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
    hole = p["depth1"] <= 0
    z = p["z1_true"]
    dm, dx = syn.epe3d(gpu, ref, z, p["cam"], hole)
    gm, gx = syn.epe3d(gpu, p["gt"], z, p["cam"], hole)
    rm, rx = syn.epe3d(ref, p["gt"], z, p["cam"], hole)
    print("hole pixels (%d): device vs reference-order oracle mean %.3g mm max %.3g mm; vs ground truth: device "
          "%.3g mm, reference order %.3g mm" % (hole.sum(), dm * 1e3, dx * 1e3, gm * 1e3, rm * 1e3))
    assert dm <= 1e-3          # the 1 mm parity bar, on hole pixels alone
    assert gm <= rm * 1.05 + 1e-4


def test_linearisation_matches_oracle(ctx):
    """One linearisation through the per-level seam (one outer iteration, no SOR iteration): the
    device's compact system against the reference's 8 planes from the oracle's linearisation of the
    same state."""
    rng = np.random.default_rng(9)
    W, H = 96, 72
    p = syn.make_pair(W=W, H=H, f=80.0, cx=47.5, cy=35.5, n_patches=3, hole_frac=0.0, seed=31)
    f1 = ob.im2feature(p["bgr1"] / 255.0)
    f2 = ob.im2feature(p["bgr2"] / 255.0)
    d1 = p["depth1"].astype(np.float64)
    d2 = p["depth2"].astype(np.float64)
    ddw = ob.stereo_error1() / ob.depth_sigma(p["depth1"]).astype(np.float64)
    dsw = np.full((H, W), 6400.0)
    mag = (80.0 / d1) ** 2
    regw = rng.uniform(0.2, 1.0, (H, W, 2))
    regw[:, -1, 0] = 0
    regw[-1, :, 1] = 0
    u0 = p["gt"][..., 0].astype(np.float64) * 0.7 + rng.normal(0, 0.05, (H, W))
    v0 = p["gt"][..., 1].astype(np.float64) * 0.7 + rng.normal(0, 0.05, (H, W))
    w0 = p["gt"][..., 2].astype(np.float64) * 0.7
    wi, wd = ob.warp(f1, d1, f2, d2, u0, v0, w0)
    cam = rf.CameraParams.make(W, H, 80.0, 47.5, 24.5)
    ctx.scene_flow_single_scale(cam, f1, d1, f2, d2, wi, wd, u0, v0, w0, 1.0, ddw, 0.02, dsw, 1e-5, mag, regw,
                                1, 1, 0, 0)
    sysd = [ctx.debug_plane(0, 0, rf.PLANE_SYSTEM, z) for z in range(12)]
    u3 = np.stack([u0, v0, w0], -1)
    A = ob.linearize(f1, d1, f2, d2, wi, wd, u3, np.zeros_like(u3), 1.0, ddw, 0.02, dsw, 1e-5, mag, regw)
    # the same linearisation from inputs rounded to FP32: how far the rounding alone moves each plane
    r = lambda x: np.asarray(x).astype(np.float32).astype(np.float64)
    wir, wdr = ob.warp(r(f1), r(d1), r(f2), r(d2), r(u0), r(v0), r(w0))
    Ar = ob.linearize(r(f1), r(d1), r(f2), r(d2), r(wir), r(wdr), r(u3), np.zeros_like(u3), 1.0, r(ddw), 0.02,
                      r(dsw), 1e-5, r(mag), r(regw))
    # the compact form's 12 planes as the reference's coefficients
    s = sysd[11]
    planes = {"diag u": (4, 0), "diag v": (5, 1), "diag w": (6, 2), "uv": (5, 0), "vu": (4, 1), "uw": (6, 0),
              "wu": (4, 2), "vw": (6, 1), "wv": (5, 2), "rhs u": (7, 0), "rhs v": (7, 1), "rhs w": (7, 2),
              "right u": (2, 0), "right w": (2, 2), "down v": (3, 1), "down w": (3, 2), "left u": (0, 0),
              "left w": (0, 2), "up v": (1, 1), "up w": (1, 2)}
    pairs = {
        "diag u": (1 / sysd[0], A[4, ..., 0]), "diag v": (1 / sysd[1], A[5, ..., 1]), "diag w": (1 / sysd[2], A[6, ..., 2]),
        "uv": (sysd[3], A[5, ..., 0]), "vu": (sysd[3], A[4, ..., 1]),
        "uw": (sysd[4], A[6, ..., 0]), "wu": (sysd[4], A[4, ..., 2]),
        "vw": (sysd[5], A[6, ..., 1]), "wv": (sysd[5], A[5, ..., 2]),
        "rhs u": (sysd[6], A[7, ..., 0]), "rhs v": (sysd[7], A[7, ..., 1]), "rhs w": (sysd[8], A[7, ..., 2]),
        "right u": (sysd[9], A[2, ..., 0]), "right w": (sysd[9] * s, A[2, ..., 2]),
        "down v": (sysd[10], A[3, ..., 1]), "down w": (sysd[10] * s, A[3, ..., 2]),
    }
    left = np.zeros((H, W)); left[:, 1:] = sysd[9][:, :-1]
    up = np.zeros((H, W)); up[1:, :] = sysd[10][:-1, :]
    sl = np.zeros((H, W)); sl[:, 1:] = s[:, :-1]
    su = np.zeros((H, W)); su[1:, :] = s[:-1, :]
    pairs["left u"] = (left, A[0, ..., 0])
    pairs["left w"] = (left * sl, A[0, ..., 2])
    pairs["up v"] = (up, A[1, ..., 1])
    pairs["up w"] = (up * su, A[1, ..., 2])
    worst, bound = {}, {}
    for name, (d, o) in pairs.items():
        pl, var = planes[name]
        worst[name] = rel(d, o)
        bound[name] = 10 * rel(Ar[pl, ..., var], o) + 1e-5
    print("linearisation (rel, bound): " + ", ".join("%s %.2g / %.2g" % (k, worst[k], bound[k]) for k in worst))
    for name in pairs:
        assert worst[name] <= bound[name], "%s: rel %.3g > %.3g" % (name, worst[name], bound[name])
