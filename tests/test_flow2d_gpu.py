"""The device 2-D optical flow (rgbdflow_optical_flow_2d, the reference demo's flow type 1) on a
B200: it keeps the reference's FP64 arithmetic, operation order and lexicographic SOR order (as
overlapping anti-diagonal sweeps), so its flow equals the reference's bit for bit (as floats,
the reference's cv::Vec2f result):
  * the golden vectors the reference made (tests/golden/ref_flow2d_golden.npz);
  * the pinned oracle on a scene where a red-black SOR order would move the flow by 1.2 px;
  * the number of sweeps in flight does not change the result."""
import importlib.util
import os

import numpy as np
import pytest

import oracle_binding as ob
import rgbdflow as rf
import synthetic as syn

pytestmark = pytest.mark.gpu

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _params(tag):
    spec = importlib.util.spec_from_file_location("make_flow2d_golden", os.path.join(GOLDEN_DIR, "make_flow2d_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    q = m.PARAMS[tag]
    return rf.flow2d_params(alpha=q["alpha"], pyramid_ratio=q["ratio"], min_width=q["min_width"], n_outer=q["n_outer"],
                            n_inner=q["n_inner"], n_sor=q["n_sor"])


@pytest.mark.parametrize("tag", ["shift", "patch"])
def test_equals_reference_golden(ctx, tag):
    g = np.load(os.path.join(GOLDEN_DIR, "ref_flow2d_golden.npz"))
    flow = ctx.optical_flow_2d(g[tag + "_bgr1"], g[tag + "_bgr2"], _params(tag))
    expect = np.stack([g[tag + "_u"], g[tag + "_v"]], -1).astype(np.float32)
    np.testing.assert_array_equal(flow, expect)


def test_equals_oracle_on_a_fragile_scene(ctx):
    p = syn.make_config_pair("160x120", seed=1)
    flow = ctx.optical_flow_2d(p["bgr1"], p["bgr2"])
    u, v = ob.optical_flow_2d(p["bgr1"], p["bgr2"])
    np.testing.assert_array_equal(flow, np.stack([u, v], -1).astype(np.float32))


def test_sweeps_in_flight_do_not_change_the_flow(ctx):
    g = np.load(os.path.join(GOLDEN_DIR, "ref_flow2d_golden.npz"))
    a = ctx.optical_flow_2d(g["patch_bgr1"], g["patch_bgr2"], _params("patch"))
    for ring in (2, 16):
        p = _params("patch")
        p.sor_ring = ring
        np.testing.assert_array_equal(ctx.optical_flow_2d(g["patch_bgr1"], g["patch_bgr2"], p), a)


def test_bad_parameters_are_status_codes(ctx):
    b = np.zeros((24, 32, 3), np.uint8)
    for over in (dict(min_width=0), dict(pyramid_ratio=0.0), dict(alpha=-1.0), dict(n_sor=0), dict(sor_ring=17)):
        with pytest.raises(rf.RgbdFlowError) as e:
            ctx.optical_flow_2d(b, b, rf.flow2d_params(**over))
        assert e.value.code == -1


@pytest.mark.parametrize("tag", ["shift", "patch"])
def test_cluster_sor_equals_reference_golden(ctx, monkeypatch, tag):
    """Every level's SOR over a cluster of CTAs with 32 sweeps in flight (the path of the larger
    levels): the same flow as the reference's, bit for bit."""
    monkeypatch.setenv("RGBDFLOW_FLOW2D_CLUSTER_MIN_PX", "1")
    g = np.load(os.path.join(GOLDEN_DIR, "ref_flow2d_golden.npz"))
    flow = ctx.optical_flow_2d(g[tag + "_bgr1"], g[tag + "_bgr2"], _params(tag))
    expect = np.stack([g[tag + "_u"], g[tag + "_v"]], -1).astype(np.float32)
    np.testing.assert_array_equal(flow, expect)


def test_cluster_sor_equals_single_cta_on_a_config_pair(ctx, monkeypatch):
    p = syn.make_config_pair("320x240", seed=2)
    monkeypatch.setenv("RGBDFLOW_FLOW2D_CLUSTER_MIN_PX", "1000000000")
    a = ctx.optical_flow_2d(p["bgr1"], p["bgr2"])
    monkeypatch.setenv("RGBDFLOW_FLOW2D_CLUSTER_MIN_PX", "1")
    b = ctx.optical_flow_2d(p["bgr1"], p["bgr2"])
    np.testing.assert_array_equal(a, b)
