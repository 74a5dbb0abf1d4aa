"""Command-line equivalent of the reference's demo driver rgbdFlowTest (src/main.cpp).

It reads two RGB-D frames: a colour PNG and an 8- or 16-bit depth PNG in millimetres for each.
It halves both frames as the demo does "for speed" and solves the forward flow on the GPU.
It can also solve the backward flow.  In the output directory it writes:
  flow0.flo3 / flow0.flo       the forward flow at the halved size: scene flow (u, v in pixels,
                               w in metres; -t 6) or 2-D flow in the Middlebury format (-t 1);
  flow0bkwd.flo3 / flow0bkwd.flo   the backward flow, with --run-bkwd 1;
  fwd-img1.png                 frame 1 as solved (halved);
  fwd-img2sampled.png          frame 2 sampled at each pixel of frame 1 moved by its flow.

Options, as in main.cpp:53-66:
  -i/--image1, -d/--depth1, -j/--image2, -e/--depth2   the two frames
  -t/--flow-type                6 = RGB-D scene flow; 1 = Ce Liu's 2-D optical flow on the
                                colour frames (runFlowTwoFramesCeLiu), which uses only -s.
                                Type 2 (2-D flow on the depth maps) stops at an assertion in the
                                reference (im2feature has no 1-channel form) and is rejected.
  -s/--smoothness-weight        default 0.02
  -v/--depth-vs-color-data-weight   default 1
  -z/--regularization-type      0 isotropic, 1 Letouzey, 2 HPB (default, as in the reference).
  --run-fwd / --run-bkwd        default 1 / 0
  -o/--outdir

The camera is the Kinect's colour camera at 640x480 (primesensor::getColorCamParams(
KINECT_640_DEFAULT), src/primesensorUtils.cpp:26-34).  The solve rescales it to the halved frames,
as runFlowTwoFramesSceneFlowExperiments does.

Image IO, the colour halving (cv::resize) and the debug image's sub-pixel sampling
(cv::getRectSubPix) go through OpenCV's Python module (cv2), as the demo's do.  For a 2-D flow the
debug image samples at (j + u, i + v); the reference reads its 2-D flow there with the stride of
a 3-channel image (flow.at<cv::Vec3f> on a cv::Vec2f matrix, main.cpp:136), which this does not
reproduce.

Run: python rgbd-flow_b200/rgbdflow_demo.py -i a.png -d a_depth.png -j b.png -e b_depth.png -t 6 -z 0 -o out
"""
import argparse
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)

import rgbdflow as rf  # noqa: E402


def _cv2():
    try:
        import cv2
    except ImportError as e:  # the demo's image IO needs OpenCV, as the reference's does
        raise SystemExit("rgbdflow_demo needs OpenCV's Python module (cv2) for PNG IO: %s" % e)
    return cv2


def kinect_640_camera():
    """primesensor::getColorCamParams(rgbd::KINECT_640_DEFAULT) (src/primesensorUtils.cpp:26-34)."""
    fov = 60 * math.pi / 180
    return rf.CameraParams(640, 480, 640 // 2, 480 // 2, 525.0, 0.072, fov, fov)


def read_depth_png(path):
    """readDepthMapValuesImg (main.cpp:31-50): an 8- or 16-bit single-channel PNG in millimetres
    -> float32 metres (value * .001 in double, stored as float)."""
    cv2 = _cv2()
    img = cv2.imread(path, cv2.IMREAD_UNCHANGED)
    if img is None:
        raise SystemExit("can't read depth image %s" % path)
    if img.ndim != 2 or img.dtype not in (np.uint8, np.uint16):
        raise SystemExit("depth image %s must be an 8- or 16-bit single-channel PNG" % path)
    return (img.astype(np.float64) * .001).astype(np.float32)


def read_color_png(path):
    """cv::imread(path) (main.cpp:110): 8-bit BGR."""
    img = _cv2().imread(path)
    if img is None:
        raise SystemExit("can't read colour image %s" % path)
    return img


def downsize_frame(img, depth):
    """downsizeFrame (src/rgbdFrameUtils.cpp:11-42) without SMOOTH_DEPTH: the colour image resized
    to (cols/2, rows/2) with cv::resize's default bilinear interpolation; depth subsampled at even
    rows and columns."""
    small = _cv2().resize(img, (img.shape[1] // 2, img.shape[0] // 2))
    h, w = depth.shape[0] // 2, depth.shape[1] // 2
    return small, np.ascontiguousarray(depth[0:2 * h:2, 0:2 * w:2])


def sample_along_flow(img2, flow):
    """The demo's fwd-img2sampled image (main.cpp:131-139): at every pixel (i, j), frame 2 sampled
    at (j + u, i + v) with cv::getRectSubPix over a 1x1 patch.  getRectSubPix replicates the border
    outside the image and is undefined for non-finite points (it crashes on some): a pixel whose
    point is not finite is black, and a point more than 4 pixels outside the image is moved to 4
    pixels outside, where it samples the same replicated border pixels."""
    cv2 = _cv2()
    H, W = flow.shape[:2]
    h2, w2 = img2.shape[:2]
    out = np.zeros((H, W, img2.shape[2]), np.uint8)
    for i in range(H):
        for j in range(W):
            x, y = float(j + flow[i, j, 0]), float(i + flow[i, j, 1])
            if not (math.isfinite(x) and math.isfinite(y)):
                continue
            x, y = min(max(x, -4.0), w2 + 3.0), min(max(y, -4.0), h2 + 3.0)
            out[i, j] = cv2.getRectSubPix(img2, (1, 1), (x, y))[0, 0]
    return out


def make_params(smoothness_weight, depth_vs_color_data_weight, regularization_type):
    """setUpSceneFlowParams (src/runFlowTwoFrames.cpp:66-100) with the demo's arguments and its
    10000 SOR iterations (main.cpp:100)."""
    p = rf.default_params()
    p.alpha = smoothness_weight
    p.depth_vs_color_data_weight = depth_vs_color_data_weight
    p.regularization = regularization_type
    p.n_sor = 10000
    return p


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description="RGB-D scene flow between two frames (rgbdFlowTest, src/main.cpp)")
    ap.add_argument("-i", "--image1", required=True, help="color image 1")
    ap.add_argument("-d", "--depth1", required=True, help="depth image 1 (16-bit png, depth in mm)")
    ap.add_argument("-j", "--image2", required=True, help="color image 2")
    ap.add_argument("-e", "--depth2", required=True, help="depth image 2 (16-bit png, depth in mm)")
    ap.add_argument("-t", "--flow-type", type=int, required=True,
                    help="6 = RGB-D scene flow; 1 = Ce Liu's 2-D optical flow")
    ap.add_argument("-s", "--smoothness-weight", type=float, default=.02)
    ap.add_argument("-v", "--depth-vs-color-data-weight", type=float, default=1.0)
    ap.add_argument("-z", "--regularization-type", type=int, default=2,
                    help="0 = isotropic; 1 = Letouzey; 2 = anisotropic from icra13 paper (HPB)")
    ap.add_argument("--run-fwd", type=int, default=1, help="whether to run forward flow")
    ap.add_argument("--run-bkwd", type=int, default=0, help="whether to run backward flow")
    ap.add_argument("-o", "--outdir", required=True)
    a = ap.parse_args(argv)
    if a.flow_type == 2:
        ap.error("flow type 2 (2-D flow on depth maps) stops at an assertion in the reference: "
                 "im2feature has no 1-channel RGB_WITH_GRADIENT form")
    if a.flow_type not in (1, 6):
        ap.error("flow type %d is not built: 1 (2-D optical flow) and 6 (RGB-D scene flow) are" % a.flow_type)
    return a


def run(args, solve=None):
    """The demo's main (main.cpp:68-150).  solve(cam, bgr1, depth1, bgr2, depth2, params) -> (H, W, 3)
    scene flow (-t 6) or (H, W, 2) 2-D flow (-t 1, params an rgbdflow.Flow2dParams); default: a
    Context's scene_flow_two_frames or optical_flow_2d on device 0."""
    cv2 = _cv2()
    os.makedirs(args.outdir, exist_ok=True)
    cam = kinect_640_camera()
    scene = args.flow_type == 6
    if scene:
        prm = make_params(args.smoothness_weight, args.depth_vs_color_data_weight, args.regularization_type)
    else:
        prm = rf.flow2d_params(alpha=args.smoothness_weight)  # runFlowTwoFramesCeLiu (runFlowTwoFrames.cpp:30-45)
    ext, write = (".flo3", rf.write_flo3) if scene else (".flo", rf.write_flo)
    ctx = None
    if solve is None:
        ctx = rf.Context(0)

        def solve(c, b1, d1, b2, d2, p):
            if scene:
                return ctx.scene_flow_two_frames(c, b1, d1, b2, d2, p, stats=False)
            return ctx.optical_flow_2d(b1, b2, p)
    try:
        prev_img, cur_img = read_color_png(args.image1), read_color_png(args.image2)
        prev_depth, cur_depth = read_depth_png(args.depth1), read_depth_png(args.depth2)
        prev_img, prev_depth = downsize_frame(prev_img, prev_depth)
        cur_img, cur_depth = downsize_frame(cur_img, cur_depth)
        written = []
        if args.run_fwd:
            t = time.perf_counter()
            flow = solve(cam, prev_img, prev_depth, cur_img, cur_depth, prm)
            print("time to call runFlowTwoFrames: %gs" % (time.perf_counter() - t))
            path = os.path.join(args.outdir, "flow0" + ext)
            write(path, flow)
            cv2.imwrite(os.path.join(args.outdir, "fwd-img1.png"), prev_img)
            cv2.imwrite(os.path.join(args.outdir, "fwd-img2sampled.png"), sample_along_flow(cur_img, flow))
            written += [path, os.path.join(args.outdir, "fwd-img1.png"), os.path.join(args.outdir, "fwd-img2sampled.png")]
        if args.run_bkwd:
            t = time.perf_counter()
            flow = solve(cam, cur_img, cur_depth, prev_img, prev_depth, prm)
            print("time to call runFlowTwoFrames: %gs" % (time.perf_counter() - t))
            path = os.path.join(args.outdir, "flow0bkwd" + ext)
            write(path, flow)
            written.append(path)
        return written
    finally:
        if ctx is not None:
            ctx.close()


def main(argv=None):
    run(parse_args(argv))
    return 0


if __name__ == "__main__":
    sys.exit(main())
