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
