"""The CPU restatement (oracle/) pinned against the reference's own code and known answers.

Runs without a GPU.  Golden vectors come from the reference's CPU image code compiled from its
sources (tests/golden/make_golden.py); where the compiled reference is present (oracle/_ref) the
oracle is also compared with it live on fresh random inputs.
"""
import os

import numpy as np
import pytest

import oracle_binding as ob
import synthetic as syn
import rgbdflow as rf

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def golden(oracle_lib):
    return np.load(os.path.join(GOLDEN, "ref_cpu_golden.npz"))


@pytest.mark.parametrize("tag", ["a", "b"])
@pytest.mark.parametrize("rtag,ratio,mw", [("r50", 0.5, 4), ("r75", 0.75, 20)])
def test_pyramid_matches_reference_golden(golden, tag, rtag, ratio, mw):
    """GaussianPyramid::ConstructPyramid (src/GaussianPyramid.cpp:20-63): bit-exact."""
    img = golden["img_" + tag]
    levels = ob.build_pyramid(img, ratio, mw)
    n = int(golden["pyr_%s_%s_n" % (tag, rtag)])
    assert len(levels) == n
    for i, lv in enumerate(levels):
        np.testing.assert_array_equal(lv, golden["pyr_%s_%s_%d" % (tag, rtag, i)])


@pytest.mark.parametrize("tag", ["a", "b"])
def test_features_resize_warp_match_reference_golden(golden, tag):
    """im2feature (OpticalFlow.cpp:189-214), Image::imresize(W,H) (Image.h:764-770) and
    warpBy3DFlow (opticalFlowUtils.cpp:76-89): bit-exact."""
    img = golden["img_" + tag]
    np.testing.assert_array_equal(ob.im2feature(img), golden["feat_" + tag])
    H, W = img.shape[:2]
    np.testing.assert_array_equal(ob.resize_dims(img[:, :, 1], 2 * W + 1, 2 * H - 1), golden["up_" + tag])
    g = {k: golden["warp_%s_%s" % (tag, k)] for k in ["f2", "d1", "d2", "u", "v", "w", "wi", "wd"]}
    wi, wd = ob.warp(golden["feat_" + tag], g["d1"], g["f2"], g["d2"], g["u"], g["v"], g["w"])
    np.testing.assert_array_equal(wi, g["wi"])
    np.testing.assert_array_equal(wd, g["wd"])


@pytest.mark.skipif(not ob.ref_cpu_available(), reason="reference CPU code not compiled (oracle/_ref)")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_matches_live_reference(seed):
    rng = np.random.default_rng(seed)
    W, H = int(rng.integers(20, 90)), int(rng.integers(15, 70))
    img = rng.random((H, W, 3))
    for ratio, mw in [(0.5, max(1, W // 16)), (0.6, 10), (0.75, 12)]:
        a = ob.build_pyramid(img, ratio, mw)
        b = ob.build_pyramid(img, ratio, mw, impl="ref")
        assert len(a) == len(b)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(ob.im2feature(img), ob.im2feature(img, impl="ref"))
    for s, fs in [(1.0, 3), (2.0, 6), (0.7, 2)]:
        np.testing.assert_array_equal(ob.gaussian_smooth(img, s, fs), ob.gaussian_smooth(img, s, fs, impl="ref"))


def test_pyramid_level_counts(oracle_lib):
    """Level count rule (GaussianPyramid.cpp:22-32): 5 levels at ratio 0.5 with minWidth = W/16."""
    for W in (160, 320, 640):
        assert oracle_lib.sfo_pyramid_levels(W, 0.5, W // 16) == 5
    assert oracle_lib.sfo_pyramid_levels(640, 0.75, 60) == 9
    # out-of-range ratios fall back to 0.75
    assert oracle_lib.sfo_pyramid_levels(640, 0.3, 60) == oracle_lib.sfo_pyramid_levels(640, 0.75, 60)


def test_median_fill_known_answers(oracle_lib):
    """recursiveMedianFilter (recursiveMedianFiltering.cpp:35-99)."""
    d = np.arange(1, 26, dtype=np.float64).reshape(5, 5)
    d[2, 2] = 0  # isolated hole: median of its 8 valid neighbours, upper median (index 4 of 8)
    out = ob.median_fill(d)
    nb = sorted([7, 8, 9, 12, 14, 17, 18, 19])
    assert out[2, 2] == nb[4]
    # corner hole: 3 neighbours
    d = np.arange(1, 17, dtype=np.float64).reshape(4, 4)
    d[0, 0] = 0
    assert ob.median_fill(d)[0, 0] == sorted([2, 5, 6])[1]
    # filled values are FP32-rounded (the reference sorts float values)
    d = np.full((3, 3), 1.0 / 3.0)
    d[1, 1] = 0
    assert ob.median_fill(d)[1, 1] == float(np.float32(1.0 / 3.0))
    # a blob fills completely, every value within the range of valid depths
    rng = np.random.default_rng(0)
    d = rng.uniform(1, 2, (20, 20))
    d[5:12, 6:10] = 0
    out = ob.median_fill(d)
    assert (out > 0).all() and out.min() >= 1 and out.max() <= 2
    # no valid depth at all is an error, as in the reference's ASSERT_ALWAYS
    with pytest.raises(RuntimeError):
        ob.median_fill(np.zeros((4, 4)))


def test_median_fill_matches_reference_golden(oracle_lib):
    """The restatement against the reference's own recursiveMedianFilterAux
    (recursiveMedianFiltering.cpp:35-99, compiled in place; tests/golden/make_rmf_golden.py): the same
    hash-set fill order, so every filled value equal."""
    g = np.load(os.path.join(GOLDEN, "ref_rmf_golden.npz"))
    for tag in ("a", "b", "c"):
        d = g["in_" + tag]
        assert (d <= 0).sum() > 0
        assert np.array_equal(ob.median_fill(d), g["out_" + tag]), tag


@pytest.mark.skipif(not ob.ref_rmf_available(), reason="reference median fill not built (oracle/_ref)")
@pytest.mark.parametrize("seed", [0, 1])
def test_median_fill_matches_live_reference(oracle_lib, seed):
    p = syn.make_config_pair("320x240", seed=seed)
    for k in ("depth1", "depth2"):
        assert np.array_equal(ob.median_fill(p[k]), ob.median_fill(p[k], impl="ref"))


def test_rounds_fill_order(oracle_lib):
    """The library's fill order (parallel rounds), restated in the oracle: isolated holes get the
    reference's value; clustered holes are all filled, each with a value taken from the valid
    depths (a median picks one of its inputs); a hole region with no valid neighbour is an error."""
    rng = np.random.default_rng(1)
    d = rng.uniform(1, 3, (30, 40))
    d[1::3, 2::3] = 0  # no two holes are 8-neighbours
    out, rounds = ob.median_fill_rounds(d)
    assert rounds == 1
    assert np.array_equal(out, ob.median_fill(d))
    p = syn.make_config_pair("320x240", seed=2)
    d = p["depth1"].astype(np.float64)
    out, rounds = ob.median_fill_rounds(d)
    assert rounds > 1 and (out > 0).all()
    assert np.isin(out[d <= 0], np.unique(d[d > 0].astype(np.float32))).all()
    with pytest.raises(RuntimeError):
        ob.median_fill_rounds(np.zeros((4, 4)))


def test_depth_sigma_matches_reference_golden(oracle_lib):
    """The restatement against the reference's own depth-noise model (staticDepthNoiseModeling.cpp:
    85-137, 225-258, compiled in place; tests/golden/make_sigma_golden.py): every sigma equal."""
    g = np.load(os.path.join(GOLDEN, "ref_sigma_golden.npz"))
    for tag in ("a", "b", "c"):
        assert np.array_equal(ob.depth_sigma(g["in_" + tag], 4), g["out_" + tag]), tag


@pytest.mark.skipif(not ob.ref_sigma_available(), reason="reference depth-noise model not built (oracle/_ref)")
@pytest.mark.parametrize("name", ["320x240", "640x480"])
def test_depth_sigma_matches_live_reference(oracle_lib, name):
    p = syn.make_config_pair(name, seed=8)
    for k in ("depth1", "depth2"):
        assert np.array_equal(ob.depth_sigma(p[k], 4), ob.depth_sigma(p[k], 4, impl="ref"))


def test_depth_sigma_known_answers(oracle_lib):
    """computeDepthMapStdevsPointwise + increaseStdevsNearDepthBoundaries
    (staticDepthNoiseModeling.cpp:232-258, 85-137)."""
    e1 = ob.stereo_error1()
    z = np.full((20, 20), 2.0, np.float32)
    s = ob.depth_sigma(z, 4)
    expect = np.float32(max(1e-4, float(np.float32(e1)) * (4 / (1 / .00285 + 2)) / e1))
    np.testing.assert_allclose(s, expect, rtol=1e-6)
    # an invalid pixel with a valid lower neighbour is itself the boundary (its min depth is 0, so
    # any difference exceeds the threshold); sigma grows by 10^(1 - d/4) within L1 distance 4
    z[10, 10] = 0
    s = ob.depth_sigma(z, 4)
    np.testing.assert_allclose(s[10, 10], 10.0, rtol=1e-5)                       # invalid: 1, d = 0
    np.testing.assert_allclose(s[9, 10], expect * 10 ** 0.75, rtol=1e-5)         # d = 1
    np.testing.assert_allclose(s[10, 12], expect * 10 ** 0.5, rtol=1e-5)         # d = 2
    np.testing.assert_allclose(s[14, 10], expect * 10 ** 0.0, rtol=1e-5)         # d = 4
    np.testing.assert_allclose(s[0, 0], expect, rtol=1e-6)                       # far away: unchanged


def _cam(p):
    c = p["cam"]
    return rf.CameraParams.make(p["W"], p["H"], c.f, c.cx, c.cy)


def test_zero_motion_gives_zero_flow(oracle_lib):
    """Identical frames: every data term's temporal derivative is 0 and the flow stays exactly 0."""
    p = syn.make_pair(W=64, H=48, f=52.5, cx=31.5, cy=23.5, n_patches=2, hole_frac=0.0, seed=3)
    prm = rf.benchmark_params(64)
    fl, st = ob.two_frames(_cam(p), p["bgr1"], p["depth1"], p["bgr1"], p["depth1"], prm)
    assert np.abs(fl).max() == 0.0


def test_oracle_recovers_synthetic_motion(oracle_lib):
    """The restated solve reduces the 2-D endpoint error far below the motion itself."""
    p = syn.make_config_pair("320x240", seed=5)
    prm = rf.benchmark_params(320)
    fl, st = ob.two_frames(_cam(p), p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
    gt, m = p["gt"], p["depth1"] > 0
    e2 = np.hypot(fl[..., 0] - gt[..., 0], fl[..., 1] - gt[..., 1])[m].mean()
    e0 = np.hypot(gt[..., 0], gt[..., 1])[m].mean()
    assert e2 < 0.25 * e0
    assert st.n_levels == 5


def test_fp64_and_faithful_variants_agree(oracle_lib):
    p = syn.make_pair(W=80, H=60, f=65.6, cx=39.5, cy=29.5, n_patches=2, hole_frac=0.03, seed=9)
    prm = rf.benchmark_params(80, fixed_schedule=1)
    a, _ = ob.two_frames(_cam(p), p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm, fp64=False)
    b, _ = ob.two_frames(_cam(p), p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm, fp64=True)
    mean, mx = syn.epe3d(a, b, p["z1_true"], p["cam"], p["depth1"] > 0)
    assert mean < 1e-5  # metres


def test_single_scale_matches_reference_cuda_golden(oracle_lib):
    """The oracle's restatement of sceneFlowSingleScale against the reference's own CUDA solver
    (outputs recorded on a B200 by make_golden.py --cuda)."""
    path = os.path.join(GOLDEN, "ref_cuda_golden.npz")
    if not os.path.exists(path):
        pytest.skip("reference CUDA golden not generated")
    g = np.load(path)
    for tag in ["s", "e"]:
        a = {k: g["%s_%s" % (tag, k)] for k in ["f1", "d1", "f2", "d2", "wi", "wd", "u", "v", "w", "ddw", "dsw", "mag", "regw"]}
        u, v, w, _, _, st = ob.single_scale(float(g[tag + "_f"]), a["f1"], a["d1"], a["f2"], a["d2"], a["wi"], a["wd"],
                                            a["u"], a["v"], a["w"], 1.0, a["ddw"], 0.02, a["dsw"], 1e-5, a["mag"],
                                            a["regw"], 4, 1, 30, int(g[tag + "_early"]))
        # FP32 system and increments: the CUDA build contracts multiply-adds (FMA), the CPU does
        # not, so agreement is to rounding (observed: 2e-6 px, 7e-8 m after 4 outer iterations)
        np.testing.assert_allclose(u, g[tag + "_out_u"], atol=2e-5)
        np.testing.assert_allclose(v, g[tag + "_out_v"], atol=2e-5)
        np.testing.assert_allclose(w, g[tag + "_out_w"], atol=1e-6)
        assert st.summary()[0][2] == (4 if tag == "s" else 1)  # outer iterations the reference ran
