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
    for t in ("1", "2", "7"):
        with pytest.raises(SystemExit):
            demo.parse_args(["-i", "a", "-d", "b", "-j", "c", "-e", "d", "-t", t, "-o", "x"])


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
