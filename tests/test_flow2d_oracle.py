"""The oracle's 2-D optical flow (Ce Liu's coarse-to-fine solver, the demo's flow type 1:
OpticalFlow::Coarse2FineFlow, src/opticalFlowMultiscale.cpp, with SmoothFlowSOR,
src/SmoothFlowSOR.cpp), pinned against the reference's own code:
  * the golden vectors of tests/golden/ref_flow2d_golden.npz (made by the reference, compiled in
    place, by tests/golden/make_flow2d_golden.py): bit-identical;
  * the reference compiled here (oracle/_ref/libref_flow2d.so), where its sources are present,
    on more seeded cases: bit-identical;
  * known answers: identical frames give exactly zero flow; a smooth texture moved by (1.5, 0.5)
    px is recovered to 0.02 px on average away from the borders.
The reference's 2-D solve is FP64 with a lexicographic SOR order, and so is the restatement.
The order a device can run in parallel and still match the reference, is checked too. It sweeps
anti-diagonal wavefronts, overlaps consecutive sweeps and keeps a ring of D flow-increment slots.
It must equal the lexicographic order bit for bit, including on a scene where a red-black order
moves the flow by more than a pixel."""
import os

import numpy as np
import pytest

import oracle_binding as ob
import synthetic as syn

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_flow2d_golden.npz")


def _golden_params():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_flow2d_golden",
                                                  os.path.join(os.path.dirname(GOLDEN), "make_flow2d_golden.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


@pytest.mark.parametrize("tag", ["shift", "patch"])
def test_oracle_equals_reference_golden(tag):
    g = np.load(GOLDEN)
    prm = _golden_params().PARAMS[tag]
    u, v = ob.optical_flow_2d(g[tag + "_bgr1"], g[tag + "_bgr2"], **prm)
    np.testing.assert_array_equal(u, g[tag + "_u"])
    np.testing.assert_array_equal(v, g[tag + "_v"])


@pytest.mark.skipif(not ob.ref_flow2d_available(), reason="reference 2-D flow not compiled (sources absent)")
@pytest.mark.parametrize("W,H,seed,prm", [
    (37, 29, 1, dict()),
    (80, 60, 2, dict(alpha=0.012, n_outer=4, n_sor=60)),
    (64, 48, 3, dict(ratio=0.5, min_width=8, n_inner=3, n_sor=25)),
])
def test_oracle_equals_reference_live(W, H, seed, prm):
    p = syn.make_pair(W=W, H=H, f=0.8 * W, cx=(W - 1) / 2, cy=(H - 1) / 2, n_patches=3, hole_frac=0.0, seed=seed)
    ur, vr = ob.optical_flow_2d(p["bgr1"], p["bgr2"], impl="ref", **prm)
    uo, vo = ob.optical_flow_2d(p["bgr1"], p["bgr2"], **prm)
    np.testing.assert_array_equal(uo, ur)
    np.testing.assert_array_equal(vo, vr)


def test_identical_frames_give_zero_flow():
    p = syn.make_pair(W=64, H=48, f=51.2, cx=31.5, cy=23.5, n_patches=3, hole_frac=0.0, seed=9)
    u, v = ob.optical_flow_2d(p["bgr1"], p["bgr1"])
    assert not np.any(u) and not np.any(v)


def test_translation_is_recovered():
    g = np.load(GOLDEN)
    u, v = ob.optical_flow_2d(g["shift_bgr1"], g["shift_bgr2"], **_golden_params().PARAMS["shift"])
    assert abs(u[8:-8, 8:-8].mean() - 1.5) < 0.02 and abs(v[8:-8, 8:-8].mean() - 0.5) < 0.02


@pytest.mark.parametrize("ring", [2, 3, 8])
def test_wavefront_order_equals_lexicographic(ring):
    g = np.load(GOLDEN)
    prm = _golden_params().PARAMS
    for tag in ("shift", "patch"):
        u0, v0 = ob.optical_flow_2d(g[tag + "_bgr1"], g[tag + "_bgr2"], **prm[tag])
        u1, v1 = ob.optical_flow_2d(g[tag + "_bgr1"], g[tag + "_bgr2"], ring=ring, **prm[tag])
        np.testing.assert_array_equal(u1, u0)
        np.testing.assert_array_equal(v1, v0)
    # a scene where a red-black sweep order moves the reference's flow by 1.2 px on average
    p = syn.make_config_pair("160x120", seed=1)
    u0, v0 = ob.optical_flow_2d(p["bgr1"], p["bgr2"])
    u1, v1 = ob.optical_flow_2d(p["bgr1"], p["bgr2"], ring=ring)
    np.testing.assert_array_equal(u1, u0)
    np.testing.assert_array_equal(v1, v0)
