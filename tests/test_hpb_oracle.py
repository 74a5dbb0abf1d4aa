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
