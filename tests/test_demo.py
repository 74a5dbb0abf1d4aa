"""The command-line equivalent of the reference's demo (rgbdflow_demo.py; src/main.cpp).

On the CPU, a recording stand-in for the solve checks everything around it:
  - the PNG reads;
  - the halving (downsizeFrame);
  - the camera and parameters;
  - the .flo3 output;
  - the debug images;
  - the backward run.
On a B200, the flow the CLI writes equals the library's solve of the same halved frames, bit for bit.
"""
import math
import os
import types

import numpy as np
import pytest

import rgbdflow as rf
import rgbdflow_demo as demo
import synthetic as syn

cv2 = pytest.importorskip("cv2")


def _write_frames(tmp_path, seed=3):
    p = syn.make_config_pair("640x480", seed=seed)
    paths = {}
    for k in ("1", "2"):
        paths["image" + k] = str(tmp_path / ("rgb%s.png" % k))
        paths["depth" + k] = str(tmp_path / ("depth%s.png" % k))
        cv2.imwrite(paths["image" + k], p["bgr" + k])
        cv2.imwrite(paths["depth" + k], np.round(p["depth" + k] * 1000.0).astype(np.uint16))
    return p, paths


def _args(paths, outdir, **over):
    argv = ["-i", paths["image1"], "-d", paths["depth1"], "-j", paths["image2"], "-e", paths["depth2"],
            "-t", "6", "-o", str(outdir)]
    for k, v in over.items():
        argv += ["--" + k.replace("_", "-"), str(v)]
    return demo.parse_args(argv)


class RecordingSolve:
    """Stands in for the GPU solve: records its inputs, returns a fixed flow of the frame's size."""

    def __init__(self, u=1.25, v=-0.75, w=0.01):
        self.calls = []
        self.uvw = (u, v, w)

    def __call__(self, cam, b1, d1, b2, d2, prm):
        self.calls.append(types.SimpleNamespace(cam=cam, b1=b1.copy(), d1=d1.copy(), b2=b2.copy(), d2=d2.copy(),
                                                prm=prm))
        flow = np.empty(d1.shape + (3,), np.float32)
        flow[...] = self.uvw
        return flow


def test_cli_around_the_solve(tmp_path):
    p, paths = _write_frames(tmp_path)
    out = tmp_path / "out"
    solve = RecordingSolve()
    written = demo.run(_args(paths, out, smoothness_weight=0.05, depth_vs_color_data_weight=2.0,
                             regularization_type=0, run_bkwd=1), solve=solve)
    assert sorted(os.path.basename(w) for w in written) == ["flow0.flo3", "flow0bkwd.flo3", "fwd-img1.png",
                                                           "fwd-img2sampled.png"]
    # the solve saw the halved frames: colour by cv::resize, depth at even rows and columns, mm -> m
    fwd, bkwd = solve.calls
    img1 = cv2.imread(paths["image1"])
    np.testing.assert_array_equal(fwd.b1, cv2.resize(img1, (320, 240)))
    mm = cv2.imread(paths["depth1"], cv2.IMREAD_UNCHANGED)
    np.testing.assert_array_equal(fwd.d1, (mm[::2, ::2].astype(np.float64) * .001).astype(np.float32))
    assert fwd.d1.shape == (240, 320) and fwd.d1.dtype == np.float32
    # backward: the same frames swapped
    np.testing.assert_array_equal(bkwd.b1, fwd.b2)
    np.testing.assert_array_equal(bkwd.d2, fwd.d1)
    # camera: the Kinect colour camera at 640x480 (the solve rescales it to the halved frames)
    c = fwd.cam
    assert (c.xRes, c.yRes, c.centerX, c.centerY, c.focalLength) == (640, 480, 320.0, 240.0, 525.0)
    assert c.fovX == pytest.approx(60 * math.pi / 180) and c.stereoBaseline == pytest.approx(0.072)
    # parameters: the reference defaults with the CLI's weights and regularisation
    assert (fwd.prm.alpha, fwd.prm.depth_vs_color_data_weight, fwd.prm.regularization) == (0.05, 2.0, 0)
    assert fwd.prm.n_sor == 10000
    # outputs
    flow = rf.read_flo3(str(out / "flow0.flo3"))
    assert flow.shape == (240, 320, 3) and np.all(flow == np.float32(solve.uvw).reshape(1, 1, 3))
    np.testing.assert_array_equal(cv2.imread(str(out / "fwd-img1.png")), fwd.b1)
    sampled = cv2.imread(str(out / "fwd-img2sampled.png"))
    u, v, _ = solve.uvw
    for i, j in [(0, 0), (10, 20), (120, 160), (239, 319)]:
        expect = cv2.getRectSubPix(fwd.b2, (1, 1), (j + u, i + v))[0, 0]
        np.testing.assert_array_equal(sampled[i, j], expect)


def test_forward_only_by_default_and_flow_types(tmp_path):
    _, paths = _write_frames(tmp_path, seed=4)
    a = _args(paths, tmp_path / "o")
    assert (a.run_fwd, a.run_bkwd, a.regularization_type, a.smoothness_weight, a.depth_vs_color_data_weight) == \
        (1, 0, 2, 0.02, 1.0)
    solve = RecordingSolve()
    written = demo.run(a, solve=solve)
    assert len(solve.calls) == 1 and not any(w.endswith("bkwd.flo3") for w in written)
    for t in ("2", "3", "7"):
        with pytest.raises(SystemExit):
            demo.parse_args(["-i", "a", "-d", "b", "-j", "c", "-e", "d", "-t", t, "-o", "x"])


class Recording2d(RecordingSolve):
    """The 2-D flow's stand-in: (H, W, 2) flow."""

    def __call__(self, cam, b1, d1, b2, d2, prm):
        self.calls.append(types.SimpleNamespace(b1=b1.copy(), b2=b2.copy(), prm=prm))
        flow = np.empty(d1.shape + (2,), np.float32)
        flow[...] = self.uvw[:2]
        return flow


def test_cli_2d_flow_type(tmp_path):
    """-t 1: Ce Liu's 2-D flow on the halved colour frames with alpha = -s, written as Middlebury
    .flo (flow0.flo, flow0bkwd.flo), and the same debug images."""
    _, paths = _write_frames(tmp_path, seed=6)
    out = tmp_path / "o2"
    solve = Recording2d(u=-0.5, v=2.25)
    argv = ["-i", paths["image1"], "-d", paths["depth1"], "-j", paths["image2"], "-e", paths["depth2"],
            "-t", "1", "-s", "0.03", "--run-bkwd", "1", "-o", str(out)]
    written = demo.run(demo.parse_args(argv), solve=solve)
    assert sorted(os.path.basename(w) for w in written) == ["flow0.flo", "flow0bkwd.flo", "fwd-img1.png",
                                                           "fwd-img2sampled.png"]
    fwd, bkwd = solve.calls
    assert fwd.prm.alpha == 0.03 and (fwd.prm.n_outer, fwd.prm.n_sor) == (10, 400)
    np.testing.assert_array_equal(fwd.b1, cv2.resize(cv2.imread(paths["image1"]), (320, 240)))
    np.testing.assert_array_equal(bkwd.b1, fwd.b2)
    flow = rf.read_flo(str(out / "flow0.flo"))
    assert flow.shape == (240, 320, 2) and np.all(flow == np.float32([-0.5, 2.25]))
    sampled = cv2.imread(str(out / "fwd-img2sampled.png"))
    np.testing.assert_array_equal(sampled[100, 100], cv2.getRectSubPix(fwd.b2, (1, 1), (99.5, 102.25))[0, 0])


def test_depth_png_must_be_single_channel(tmp_path):
    p = tmp_path / "rgb_as_depth.png"
    cv2.imwrite(str(p), np.zeros((4, 4, 3), np.uint8))
    with pytest.raises(SystemExit):
        demo.read_depth_png(str(p))
    q = tmp_path / "d8.png"
    cv2.imwrite(str(q), np.full((4, 4), 200, np.uint8))
    np.testing.assert_array_equal(demo.read_depth_png(str(q)), np.float32(0.2))


@pytest.mark.gpu
def test_cli_flow_equals_the_library_solve(tmp_path, ctx):
    _, paths = _write_frames(tmp_path, seed=5)
    out = tmp_path / "out"
    demo.run(_args(paths, out, regularization_type=0))
    flow = rf.read_flo3(str(out / "flow0.flo3"))
    b1, d1 = demo.downsize_frame(demo.read_color_png(paths["image1"]), demo.read_depth_png(paths["depth1"]))
    b2, d2 = demo.downsize_frame(demo.read_color_png(paths["image2"]), demo.read_depth_png(paths["depth2"]))
    direct = ctx.scene_flow_two_frames(demo.kinect_640_camera(), b1, d1, b2, d2, demo.make_params(0.02, 1.0, 0),
                                       stats=False)
    assert flow.shape == (240, 320, 3) and np.isfinite(flow).all()
    np.testing.assert_array_equal(flow, direct)


def _write_textured_shift(tmp_path):
    """A smooth random texture moved by (3, 1) px, 144x112 (72x56 once halved), with a flat depth:
    a well-posed 2-D flow (on the synthetic patch scenes the reference's 2-D solver diverges)."""
    rng = np.random.default_rng(12)
    t = rng.random((140, 172, 3))
    for _ in range(3):
        t = sum(np.roll(np.roll(t, dy, 0), dx, 1) for dy in range(-2, 3) for dx in range(-2, 3)) / 25
    t = (t - t.min()) / (t.max() - t.min()) * 255
    paths = {}
    for k, (dy, dx) in (("1", (0, 0)), ("2", (1, 3))):
        img = np.rint(np.roll(np.roll(t, dy, 0), dx, 1)[14:126, 14:158]).astype(np.uint8)
        paths["image" + k] = str(tmp_path / ("t%s.png" % k))
        paths["depth" + k] = str(tmp_path / ("td%s.png" % k))
        cv2.imwrite(paths["image" + k], img)
        cv2.imwrite(paths["depth" + k], np.full(img.shape[:2], 1500, np.uint16))
    return paths


def test_debug_image_survives_non_finite_and_far_points():
    img = np.arange(4 * 5 * 3, dtype=np.uint8).reshape(4, 5, 3)
    flow = np.zeros((4, 5, 2), np.float32)
    flow[0, 0] = (np.nan, 0)
    flow[1, 1] = (1e30, -1e30)
    flow[2, 2] = (-3e9, 0.25)
    out = demo.sample_along_flow(img, flow)
    assert not out[0, 0].any()
    np.testing.assert_array_equal(out[1, 1], cv2.getRectSubPix(img, (1, 1), (4 + 3.0, -4.0))[0, 0])
    np.testing.assert_array_equal(out[2, 2], cv2.getRectSubPix(img, (1, 1), (-4.0, 2.25))[0, 0])
    np.testing.assert_array_equal(out[3, 4], img[3, 4])


@pytest.mark.gpu
def test_cli_2d_flow_equals_the_library_solve(tmp_path, ctx):
    paths = _write_textured_shift(tmp_path)
    out = tmp_path / "o"
    demo.run(demo.parse_args(["-i", paths["image1"], "-d", paths["depth1"], "-j", paths["image2"], "-e",
                              paths["depth2"], "-t", "1", "-o", str(out)]))
    b1, _ = demo.downsize_frame(demo.read_color_png(paths["image1"]), demo.read_depth_png(paths["depth1"]))
    b2, _ = demo.downsize_frame(demo.read_color_png(paths["image2"]), demo.read_depth_png(paths["depth2"]))
    flow = rf.read_flo(str(out / "flow0.flo"))
    assert flow.shape == (56, 72, 2) and np.isfinite(flow).all()
    assert abs(flow[8:-8, 8:-8, 0].mean() - 1.5) < 0.1 and abs(flow[8:-8, 8:-8, 1].mean() - 0.5) < 0.1
    np.testing.assert_array_equal(flow, ctx.optical_flow_2d(b1, b2))
