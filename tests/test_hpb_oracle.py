"""The oracle's restatement of the HPB regularisation's raw-depth pyramid
(DepthMapPyramid::ConstructPyramid, src/depthMapPyramid.cpp:15-91), pinned against the
reference's own code:
  * the golden vectors of tests/golden/ref_hpb_golden.npz (made by the reference, compiled in
    place, by tests/golden/make_hpb_golden.py): bit-identical;
  * the reference compiled here (oracle/_ref/libref_hpb.so), where its sources are present, on
    the synthetic scene depth maps of every configuration: bit-identical.
The rest of HPB (normals from PCL, a Boost-hash-ordered depth fill) cannot be pinned; this part
can."""
import os

import numpy as np
import pytest

import oracle_binding as ob
import synthetic as syn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_hpb_golden.npz")


@pytest.mark.parametrize("tag,ratio,mw", [("r75", 0.75, 20), ("r50", 0.5, 10)])
def test_depth_pyramid_equals_reference_golden(tag, ratio, mw):
    g = np.load(GOLDEN)
    levels = ob.depth_map_pyramid(g["depth"], ratio, mw)
    assert len(levels) == int(g[tag + "_n"])
    for i, lv in enumerate(levels):
        np.testing.assert_array_equal(lv, g["%s_%d" % (tag, i)])


@pytest.mark.skipif(not ob.ref_hpb_available(), reason="reference DepthMapPyramid not compiled (sources absent)")
@pytest.mark.parametrize("name,seed", [("160x120", 1), ("320x240", 2), ("640x480", 3)])
@pytest.mark.parametrize("ratio,mw", [(0.75, 20), (0.5, 10)])
def test_depth_pyramid_equals_reference_live(name, seed, ratio, mw):
    d = syn.make_config_pair(name, seed=seed)["depth1"]
    a = ob.depth_map_pyramid(d, ratio, mw, impl="ref")
    b = ob.depth_map_pyramid(d, ratio, mw)
    assert len(a) == len(b)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(y, x)


def test_invalid_depth_stays_invalid_and_flat_depth_stays_flat():
    d = np.full((40, 60), 2.0)
    d[10:14, 20:30] = 0
    levels = ob.depth_map_pyramid(d, 0.5, 10)
    assert np.all((levels[1] == 2.0) | (levels[1] == -1)) and (levels[1] == -1).any()
    assert np.all(ob.depth_map_pyramid(np.full((40, 60), 1.25), 0.5, 10)[-1] == 1.25)


# computeHeuristicPb on one level (heuristicBoundaries.cpp:40-358), known answers on 60x40 levels
_H, _W = 40, 60


def _grey():
    return np.full((_H, _W, 3), 0.5)


def test_hpb_flat_plane_has_no_boundary():
    assert ob.heuristic_pb(_grey(), np.full((_H, _W), 1.5)).max() == 0


def test_hpb_depth_step_is_a_boundary_on_the_straddling_pair_only():
    d = np.full((_H, _W), 2.0)
    d[:, :30] = 1.0
    pb = ob.heuristic_pb(_grey(), d)
    np.testing.assert_array_equal(pb[:, 29, 0], 1.0)
    assert np.delete(pb[..., 0], 29, axis=1).max() == 0 and pb[..., 1].max() == 0


def test_hpb_invalid_run_length_follows_the_reference_search():
    """Next to invalid depth the probability is linterp(.2, 1, run / 30), the run counted from
    the invalid pixel of the pair, or from the pixel before the valid one (heuristicBoundaries.cpp:
    239-252: the start offset uses the direction code of the pair, not its neighbour)."""
    d = np.full((_H, _W), 1.5)
    d[:, 20:25] = 0
    pb = ob.heuristic_pb(_grey(), d)
    assert pb[10, 19, 0] == np.float32(0.2)
    assert pb[10, 24, 0] == np.float32((1 - 1 / 30) * .2 + 1 / 30)


def test_hpb_colour_edge_without_depth():
    """Without valid depth only colour counts: 1 - exp(-(dcol / .7)^2) at the edge, after the
    8-bit truncation of the level image (heuristicProbBoundary.cpp:33)."""
    img = _grey()
    img[:, 30:] = 0.9
    pb = ob.heuristic_pb(img, np.zeros((_H, _W)))
    a, b = int(255 * 0.5) / 255.0, int(255 * 0.9) / 255.0
    expect = np.float32(1 - np.exp(-((np.sqrt(3) * (np.float32(b) - np.float32(a))) / np.float32(0.7)) ** 2))
    assert set(np.argmax(pb[..., 0], axis=1)) == {29}
    # the half-disk means come from float integral images, as in the reference; their
    # cancellation error grows with the row (2e-5 at the bottom of this level)
    assert abs(pb[:, 29, 0] - expect).max() < 1e-4


def test_colour_guided_fill_known_answers():
    """recursiveMedianFilterSmallInvalidRegionsUsingColor (recursiveMedianFiltering.cpp:127-222):
    a hole in constant depth takes that depth; the colour weights pull a hole towards the side of
    its own colour; a region larger than the limit stays invalid."""
    col = np.full((20, 30, 3), 0.5)
    d = np.full((20, 30), 2.0)
    d[5, 5] = 0
    d[10:12, 10:13] = 0
    out = ob.fill_small_regions_color(d, col)
    np.testing.assert_array_equal(out, np.full((20, 30), 2.0))
    d = np.full((20, 30), 1.0)
    d[:, 15:] = 3.0
    col2 = col.copy()
    col2[:, 15:] = 0.9
    d[8, 15] = 0  # a hole on the 3 m side, whose colour it shares
    out = ob.fill_small_regions_color(d, col2)
    # 3 neighbours at 1 m of the other colour (weight exp(-3 * .4^2 / .6)), 5 at 3 m of its own (weight 1)
    w = np.exp(-3 * (0.9 - 0.5) ** 2 / 0.6)
    assert abs(out[8, 15] - (3 * w * 1.0 + 5 * 3.0) / (3 * w + 5)) < 1e-5
    d = np.full((20, 30), 2.0)
    d[2:12, 2:12] = 0  # 100 pixels > 60
    out = ob.fill_small_regions_color(d, col)
    assert np.all(out[2:12, 2:12] == 0) and np.all(out[:2] == 2.0)


def test_hpb_scene_flow_end_to_end():
    """The oracle's scene flow with HPB regularisation (per level: colour-guided fill of the raw
    depth, DepthMapPyramid, computeHeuristicPb, weights 1 - .99 hpb) is finite and no less accurate
    against ground truth than the isotropic solve on a textured-patch scene."""
    import rgbdflow as rf
    p = syn.make_config_pair("320x240", seed=3)
    cam = rf.CameraParams.make(p["W"], p["H"], p["cam"].f, p["cam"].cx, p["cam"].cy)
    iso = rf.benchmark_params(320)
    hpb = rf.benchmark_params(320)
    hpb.regularization = rf.REG_HPB
    fi, _ = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], iso)
    fh, _ = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], hpb)
    assert np.isfinite(fh).all() and not np.array_equal(fh, fi)
    valid = p["depth1"] > 0
    ei = syn.epe3d(fi, p["gt"], p["z1_true"], p["cam"], valid)[0]
    eh = syn.epe3d(fh, p["gt"], p["z1_true"], p["cam"], valid)[0]
    assert eh <= ei * 1.05


def test_depth_map_pyramid_min_width_conventions(oracle_lib):
    """A negative min_width is the library's W / d convention; 0 never ends the level count and is
    an error (the reference loops for ever)."""
    d = np.full((48, 64), 2.0)
    a = ob.depth_map_pyramid(d, 0.5, -16)
    b = ob.depth_map_pyramid(d, 0.5, 4)
    assert [x.shape for x in a] == [x.shape for x in b]
    with pytest.raises(RuntimeError):
        ob.depth_map_pyramid(d, 0.5, 0)
    with pytest.raises(RuntimeError):
        ob.build_pyramid(d, 0.5, 0)
