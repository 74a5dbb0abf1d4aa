"""ctypes bindings of the CPU restatement (oracle/libsforacle.so) and of the reference's own
code compiled in place (oracle/_ref/libref_cpu.so, oracle/_ref/libref_cuda.so,
oracle/_ref/libref_flow2d.so).

Test infrastructure only: the checker side of the parity tests, the smoke check and the CPU
baseline of the benchmark.  The product path never imports this module.
"""
import ctypes
import os
import sys
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "libsforacle.so")
REF_CPU_SO = os.path.join(ORACLE_DIR, "_ref", "libref_cpu.so")
REF_CUDA_SO = os.path.join(ORACLE_DIR, "_ref", "libref_cuda.so")
REF_FLOW2D_SO = os.path.join(ORACLE_DIR, "_ref", "libref_flow2d.so")
REF_RMF_SO = os.path.join(ORACLE_DIR, "_ref", "libref_rmf.so")
REF_HPB_SO = os.path.join(ORACLE_DIR, "_ref", "libref_hpb.so")

_P = ctypes.POINTER
_d = ctypes.c_double
_i = ctypes.c_int
_f = ctypes.c_float
_pd = _P(ctypes.c_double)
_pf = _P(ctypes.c_float)
_pi = _P(ctypes.c_int)
_pu8 = _P(ctypes.c_uint8)


def build_oracle():
    """Compile the oracle (and, where the reference sources exist, oracle/_ref) with make."""
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def dptr(a):
    return a.ctypes.data_as(_pd)


def fptr(a):
    return a.ctypes.data_as(_pf)


def iptr(a):
    return a.ctypes.data_as(_pi)


def u8ptr(a):
    return a.ctypes.data_as(_pu8)


def _cont(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.sfo_pyramid_levels.argtypes = [_i, _d, _i]
        lib.sfo_build_pyramid.argtypes = [_pd, _i, _i, _i, _d, _i, _pd, _pi]
        lib.sfo_gaussian_smooth.argtypes = [_pd, _i, _i, _i, _d, _i, _pd]
        lib.sfo_resize_dims.argtypes = [_pd, _i, _i, _i, _i, _i, _pd]
        lib.sfo_im2feature.argtypes = [_pd, _i, _i, _pd]
        lib.sfo_median_fill.argtypes = [_pd, _i, _i]
        lib.sfo_median_fill_rounds.argtypes = [_pd, _i, _i, _pi]
        lib.sfo_set_fill_order.argtypes = [_i]
        lib.sfo_set_level_solver.argtypes = [ctypes.c_void_p]
        lib.sfo_depth_sigma.argtypes = [_pf, _i, _i, _i, _pf]
        lib.sfo_warp_cpu.argtypes = [_pd, _pd, _pd, _pd, _i, _i, _i, _pd, _pd, _pd, _pd, _pd]
        lib.sfo_depth_mag_weights.argtypes = [_pd, _i, _i, ctypes.c_void_p, _pd]
        lib.sfo_reg_weights.argtypes = [_pd, _i, _i, _i, _pd]
        lib.sfo_linearize.argtypes = [_i] + [_pd] * 8 + [_i, _i, _i, _d, _pd, _d, _pd, _d, _pd, _pd, ctypes.c_void_p, _pd]
        lib.sfo_sor.argtypes = [_i, _pd, _pd, _i, _i, _i, _d, _d]
        lib.sfo_single_scale.argtypes = ([_i, _f] + [_pd] * 9 + [_i, _i, _i, _d, _pd, _d, _pd, _d, _pd, _pd,
                                         _i, _i, _i, _i, ctypes.c_void_p, ctypes.c_void_p])
        lib.sfo_scene_flow_two_frames.argtypes = [_i, ctypes.c_void_p, _pu8, _pf, _pu8, _pf, _i, _i,
                                                  ctypes.c_void_p, _pf, _pf, ctypes.c_void_p]
        lib.sfo_optical_flow_2d.argtypes = [_pu8, _pu8, _i, _i, _d, _d, _i, _i, _i, _i, _pd, _pd]
        lib.sfo_optical_flow_2d_ring.argtypes = [_pu8, _pu8, _i, _i, _d, _d, _i, _i, _i, _i, _i, _pd, _pd]
        lib.sfo_depth_map_pyramid.argtypes = [_pd, _i, _i, _d, _i, _pd, _pi]
        lib.sfo_heuristic_pb.argtypes = [_pd, _pd, _i, _i, _pf]
        lib.sfo_fill_small_regions_color.argtypes = [_pd, _pd, _i, _i, _i]
        lib.sfo_last_error.restype = ctypes.c_char_p
        lib.sfo_set_threads.argtypes = [_i]
        _oracle = lib
    return _oracle


_ref_cpu = None


def ref_cpu_available():
    return os.path.exists(REF_CPU_SO)


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        lib = ctypes.CDLL(REF_CPU_SO)
        lib.ref_build_pyramid.argtypes = [_pd, _i, _i, _i, _d, _i, _pd, _pi]
        lib.ref_gaussian_smooth.argtypes = [_pd, _i, _i, _i, _d, _i, _pd]
        lib.ref_resize_dims.argtypes = [_pd, _i, _i, _i, _i, _i, _pd]
        lib.ref_im2feature.argtypes = [_pd, _i, _i, _pd]
        lib.ref_warp.argtypes = [_pd, _pd, _pd, _pd, _i, _i, _i, _pd, _pd, _pd, _pd, _pd]
        _ref_cpu = lib
    return _ref_cpu


_ref_cuda = None


def ref_cuda_available():
    return os.path.exists(REF_CUDA_SO)


def ref_cuda():
    global _ref_cuda
    if _ref_cuda is None:
        lib = ctypes.CDLL(REF_CUDA_SO)
        lib.ref_single_scale.argtypes = ([_f] + [_pd] * 9 + [_i, _i, _i, _d, _pd, _d, _pd, _d, _pd, _pd, _i, _i, _i, _i])
        _ref_cuda = lib
    return _ref_cuda


_ref_flow2d = None


def ref_flow2d_available():
    return os.path.exists(REF_FLOW2D_SO)


def ref_flow2d():
    global _ref_flow2d
    if _ref_flow2d is None:
        lib = ctypes.CDLL(REF_FLOW2D_SO)
        lib.ref_coarse2fine_flow.argtypes = [_pd, _pd, _i, _i, _i, _d, _d, _i, _i, _i, _i, _pd, _pd,
                                             ctypes.c_char_p, _i]
        _ref_flow2d = lib
    return _ref_flow2d


def optical_flow_2d(bgr1, bgr2, alpha=0.02, ratio=0.75, min_width=20, n_outer=10, n_inner=1, n_sor=400,
                    impl="oracle", ring=0):
    """2-D optical flow (u, v) of two (H, W, 3) uint8 BGR images: the demo's flow type 1 with its
    defaults (runFlowTwoFramesCeLiu, src/runFlowTwoFrames.cpp:30-45; opticalFlowParams ratio
    0.75, minWidth 20).  impl "oracle" (the restatement) or "ref" (the reference, compiled).
    ring > 0 (oracle only): the SOR iterations in the device order, anti-diagonal wavefronts
    with overlapping sweeps and a ring of that many slots."""
    b1, b2 = _cont(bgr1, np.uint8), _cont(bgr2, np.uint8)
    H, W = b1.shape[:2]
    u = np.zeros((H, W)); v = np.zeros((H, W))
    if impl == "ref":
        d1, d2 = b1.astype(np.float64) / 255.0, b2.astype(np.float64) / 255.0
        err = ctypes.create_string_buffer(256)
        rc = ref_flow2d().ref_coarse2fine_flow(dptr(d1), dptr(d2), W, H, 0, alpha, ratio, min_width, n_outer, n_inner,
                                               n_sor, dptr(u), dptr(v), err, len(err))
        if rc != 0:
            raise RuntimeError("reference Coarse2FineFlow: " + err.value.decode())
    else:
        rc = oracle().sfo_optical_flow_2d_ring(u8ptr(b1), u8ptr(b2), W, H, alpha, ratio, min_width, n_outer, n_inner,
                                               n_sor, ring, dptr(u), dptr(v))
        if rc != 0:
            raise RuntimeError("oracle 2-D flow: " + oracle().sfo_last_error().decode())
    return u, v


_ref_hpb = None


def fill_small_regions_color(depth, col, max_region=60):
    """recursiveMedianFilterSmallInvalidRegionsUsingColor (oracle, deterministic order): a filled
    copy of depth (H, W), guided by col (H, W, 3) in [0, 1]."""
    d, c = _cont(depth, np.float64).copy(), _cont(col, np.float64)
    H, W = d.shape
    if oracle().sfo_fill_small_regions_color(dptr(d), dptr(c), W, H, max_region) != 0:
        raise RuntimeError(oracle().sfo_last_error().decode())
    return d


def heuristic_pb(img, depth):
    """computeHeuristicPb of one pyramid level (oracle): img (H, W, 3) in [0, 1] (BGR), depth
    (H, W) metres (<= 0 invalid) -> (H, W, 2) float32 boundary probabilities (right, down)."""
    im, d = _cont(img, np.float64), _cont(depth, np.float64)
    H, W = d.shape
    out = np.zeros((H, W, 2), np.float32)
    oracle().sfo_heuristic_pb(dptr(im), dptr(d), W, H, fptr(out))
    return out


def ref_hpb_available():
    return os.path.exists(REF_HPB_SO)


def depth_map_pyramid(depth, ratio, min_width, impl="oracle"):
    """DepthMapPyramid::ConstructPyramid (src/depthMapPyramid.cpp:15-91) of a depth map: the list
    of levels.  impl "oracle" (the restatement) or "ref" (the reference, compiled)."""
    global _ref_hpb
    d = _cont(depth, np.float64)
    H, W = d.shape
    if impl == "ref":
        if _ref_hpb is None:
            _ref_hpb = ctypes.CDLL(REF_HPB_SO)
            _ref_hpb.ref_depth_map_pyramid.argtypes = [_pd, _i, _i, _d, _i, _pd, _pi]
        fn = _ref_hpb.ref_depth_map_pyramid
    else:
        fn = oracle().sfo_depth_map_pyramid
    dims = np.zeros(128, np.int32)
    n = fn(dptr(d), W, H, ratio, min_width, None, iptr(dims))
    if n < 0:
        raise RuntimeError(oracle().sfo_last_error().decode())
    out = np.zeros(sum(int(dims[2 * i]) * int(dims[2 * i + 1]) for i in range(n)))
    fn(dptr(d), W, H, ratio, min_width, dptr(out), iptr(dims))
    levels, off = [], 0
    for i in range(n):
        w, h = int(dims[2 * i]), int(dims[2 * i + 1])
        levels.append(out[off:off + w * h].reshape(h, w))
        off += w * h
    return levels


# ---------------------------------------------------------------------------------------------
# numpy-level helpers over either implementation ("oracle" or "ref")

def build_pyramid(img, ratio, min_width, impl="oracle"):
    img = _cont(img, np.float64)
    H, W = img.shape[:2]
    C = 1 if img.ndim == 2 else img.shape[2]
    lib = oracle() if impl == "oracle" else ref_cpu()
    fn = lib.sfo_build_pyramid if impl == "oracle" else lib.ref_build_pyramid
    dims = np.zeros(64, np.int32)
    n = fn(dptr(img), W, H, C, ratio, min_width, None, iptr(dims))
    if n < 0:
        raise RuntimeError(oracle().sfo_last_error().decode())
    total = sum(int(dims[2 * i]) * int(dims[2 * i + 1]) * C for i in range(n))
    out = np.zeros(total, np.float64)
    fn(dptr(img), W, H, C, ratio, min_width, dptr(out), iptr(dims))
    levels, off = [], 0
    for i in range(n):
        w, h = int(dims[2 * i]), int(dims[2 * i + 1])
        shape = (h, w) if C == 1 else (h, w, C)
        levels.append(out[off:off + w * h * C].reshape(shape).copy())
        off += w * h * C
    return levels


def gaussian_smooth(img, sigma, fsize, impl="oracle"):
    img = _cont(img, np.float64)
    H, W = img.shape[:2]
    C = 1 if img.ndim == 2 else img.shape[2]
    out = np.zeros_like(img)
    if impl == "oracle":
        oracle().sfo_gaussian_smooth(dptr(img), W, H, C, sigma, fsize, dptr(out))
    else:
        ref_cpu().ref_gaussian_smooth(dptr(img), W, H, C, sigma, fsize, dptr(out))
    return out


def resize_dims(img, DW, DH, impl="oracle"):
    img = _cont(img, np.float64)
    H, W = img.shape[:2]
    C = 1 if img.ndim == 2 else img.shape[2]
    out = np.zeros((DH, DW) if C == 1 else (DH, DW, C), np.float64)
    fn = oracle().sfo_resize_dims if impl == "oracle" else ref_cpu().ref_resize_dims
    fn(dptr(img), W, H, C, DW, DH, dptr(out))
    return out


def im2feature(bgr01, impl="oracle"):
    bgr01 = _cont(bgr01, np.float64)
    H, W = bgr01.shape[:2]
    out = np.zeros((H, W, 5), np.float64)
    fn = oracle().sfo_im2feature if impl == "oracle" else ref_cpu().ref_im2feature
    fn(dptr(bgr01), W, H, dptr(out))
    return out


def warp(feat1, d1, feat2, d2, u, v, w, impl="oracle"):
    feat1, feat2 = _cont(feat1, np.float64), _cont(feat2, np.float64)
    d1, d2 = _cont(d1, np.float64), _cont(d2, np.float64)
    u, v, w = _cont(u, np.float64), _cont(v, np.float64), _cont(w, np.float64)
    H, W, C = feat1.shape
    wI = np.zeros_like(feat1)
    wD = np.zeros_like(d1)
    fn = oracle().sfo_warp_cpu if impl == "oracle" else ref_cpu().ref_warp
    fn(dptr(feat1), dptr(d1), dptr(feat2), dptr(d2), W, H, C, dptr(u), dptr(v), dptr(w), dptr(wI), dptr(wD))
    return wI, wD


_ref_rmf = None


def ref_rmf_available():
    return os.path.exists(REF_RMF_SO)


def median_fill(depth, impl="oracle"):
    """recursiveMedianFilter, the restatement (impl="oracle") or the reference's own code compiled in
    place (impl="ref", oracle/_ref/libref_rmf.so)."""
    global _ref_rmf
    d = _cont(depth, np.float64).copy()
    H, W = d.shape
    if impl == "ref":
        if _ref_rmf is None:
            _ref_rmf = ctypes.CDLL(REF_RMF_SO)
            _ref_rmf.ref_median_fill.argtypes = [_pd, _i, _i]
            _ref_rmf.ref_median_fill.restype = None
        _ref_rmf.ref_median_fill(dptr(d), W, H)
        return d
    rc = oracle().sfo_median_fill(dptr(d), W, H)
    if rc != 0:
        raise RuntimeError(oracle().sfo_last_error().decode())
    return d


def median_fill_rounds(depth):
    """The hole fill in the library's order (parallel rounds); returns (filled depth, rounds)."""
    d = _cont(depth, np.float64).copy()
    H, W = d.shape
    r = ctypes.c_int(0)
    rc = oracle().sfo_median_fill_rounds(dptr(d), W, H, ctypes.byref(r))
    if rc != 0:
        raise RuntimeError(oracle().sfo_last_error().decode())
    return d, r.value


class reference_cuda_levels:
    """Context manager: the oracle's faithful scene-flow solves hand every pyramid level to the
    reference's own CUDA solver (oracle/_ref/libref_cuda.so, needs a GPU), as the reference's
    sceneFlowMultiscale does; pyramids, features, warps and weights stay on the host."""

    def __enter__(self):
        fn = ctypes.cast(ref_cuda().ref_single_scale, ctypes.c_void_p).value
        oracle().sfo_set_level_solver(fn)
        # the reference solver prints its timings on stdout: sent to stderr while it runs, so that
        # a caller's stdout (bench.py's one JSON line) stays clean
        sys.stdout.flush()
        self._stdout = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *a):
        ctypes.CDLL(None).fflush(None)
        os.dup2(self._stdout, 1)
        os.close(self._stdout)
        oracle().sfo_set_level_solver(None)


class fill_order:
    """Context manager: the oracle's scene-flow solves fill holes in the given order ("reference":
    the reference's hash-set order; "rounds": the library's parallel rounds)."""

    def __init__(self, order):
        self.order = {"reference": 0, "rounds": 1}[order]

    def __enter__(self):
        self.old = oracle().sfo_set_fill_order(self.order)
        return self

    def __exit__(self, *a):
        oracle().sfo_set_fill_order(self.old)


REF_SIGMA_SO = os.path.join(ORACLE_DIR, "_ref", "libref_sigma.so")
_ref_sigma = None


def ref_sigma_available():
    return os.path.exists(REF_SIGMA_SO)


def depth_sigma(depth_m, max_dist=4, impl="oracle"):
    """The depth sigma of setUpSceneFlowParams: the restatement (impl="oracle") or the reference's own
    depth-noise model compiled in place (impl="ref", oracle/_ref/libref_sigma.so)."""
    global _ref_sigma
    d = _cont(depth_m, np.float32)
    H, W = d.shape
    out = np.zeros_like(d)
    if impl == "ref":
        if _ref_sigma is None:
            _ref_sigma = ctypes.CDLL(REF_SIGMA_SO)
            _ref_sigma.ref_depth_sigma.argtypes = [_pf, _i, _i, _i, _pf]
            _ref_sigma.ref_depth_sigma.restype = None
        _ref_sigma.ref_depth_sigma(fptr(d), W, H, max_dist, fptr(out))
        return out
    oracle().sfo_depth_sigma(fptr(d), W, H, max_dist, fptr(out))
    return out


def two_frames(cam, bgr1, depth1, bgr2, depth2, params, fp64=False, est_flow=None):
    """sfo_scene_flow_two_frames: returns ((H,W,3) float32 flow, Stats).  cam and params are the
    ctypes structs of the product binding (rgbdflow.CameraParams / rgbdflow.Params)."""
    import rgbdflow as rf
    bgr1, bgr2 = _cont(bgr1, np.uint8), _cont(bgr2, np.uint8)
    depth1, depth2 = _cont(depth1, np.float32), _cont(depth2, np.float32)
    H, W = depth1.shape
    out = np.zeros((H, W, 3), np.float32)
    st = rf.Stats()
    est = _cont(est_flow, np.float32) if est_flow is not None else None
    rc = oracle().sfo_scene_flow_two_frames(int(fp64), ctypes.byref(cam), u8ptr(bgr1), fptr(depth1), u8ptr(bgr2),
                                            fptr(depth2), W, H, ctypes.byref(params),
                                            fptr(est) if est is not None else None, fptr(out), ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle: %s" % oracle().sfo_last_error().decode())
    return out, st


def depth_mag_weights(depth_k, cam_full):
    """calculateDepthMagnitudeTermWeights at a level, with the reference's full-resolution indexing."""
    d = _cont(depth_k, np.float64)
    H, W = d.shape
    out = np.zeros((H, W), np.float64)
    oracle().sfo_depth_mag_weights(dptr(d), W, H, ctypes.byref(cam_full), dptr(out))
    return out


def reg_weights(depth, reg_type):
    """calculateRegularizationWeights (ISOTROPIC / LETOUZEY): (H, W, 2) right / down weights."""
    d = _cont(depth, np.float64)
    H, W = d.shape
    out = np.zeros((H, W, 2), np.float64)
    oracle().sfo_reg_weights(dptr(d), W, H, reg_type, dptr(out))
    return out


def linearize(Im1, dm1, Im2, dm2, wI2, wD2, u3, du3, colorW, ddw, alpha, dsw, gamma, mag, regw, params=None,
              fp64=False):
    """One linearisation (fillSystemMtxKernel and the kernels before it, .cu:84-575) from the state
    (u3, du3: (H, W, 3)); returns the reference's 8 system planes as an (8, H, W, 3) array."""
    Im1, Im2 = _cont(Im1, np.float64), _cont(Im2, np.float64)
    dm1, dm2, wI2, wD2 = (_cont(x, np.float64) for x in (dm1, dm2, wI2, wD2))
    u3, du3 = _cont(u3, np.float64), _cont(du3, np.float64)
    ddw, dsw, mag, regw = (_cont(x, np.float64) for x in (ddw, dsw, mag, regw))
    H, W, C = Im1.shape
    A = np.zeros((8, H, W, 3), np.float64)
    rc = oracle().sfo_linearize(int(fp64), dptr(Im1), dptr(dm1), dptr(Im2), dptr(dm2), dptr(wI2), dptr(wD2),
                                dptr(u3), dptr(du3), W, H, C, colorW, dptr(ddw), alpha, dptr(dsw), gamma, dptr(mag),
                                dptr(regw), ctypes.byref(params) if params is not None else None, dptr(A))
    if rc != 0:
        raise RuntimeError("oracle: %s" % oracle().sfo_last_error().decode())
    return A


def single_scale(f_level, Im1, dm1, Im2, dm2, wI2, wD2, u, v, w, colorW, ddw, alpha, dsw, gamma, mag, regw,
                 nOuter, nInner, nSOR, allowEarly, params=None, fp64=False, impl="oracle"):
    """The per-level seam on the oracle (impl="oracle") or on the reference's own CUDA solver
    (impl="ref", needs a GPU).  Returns (u, v, w, warpIm2, warpDm2, stats-or-None)."""
    import rgbdflow as rf
    Im1, Im2 = _cont(Im1, np.float64), _cont(Im2, np.float64)
    dm1, dm2 = _cont(dm1, np.float64), _cont(dm2, np.float64)
    wI2, wD2 = _cont(wI2, np.float64).copy(), _cont(wD2, np.float64).copy()
    u, v, w = _cont(u, np.float64).copy(), _cont(v, np.float64).copy(), _cont(w, np.float64).copy()
    ddw, dsw, mag, regw = (_cont(x, np.float64) for x in (ddw, dsw, mag, regw))
    H, W, C = Im1.shape
    if impl == "ref":
        rc = ref_cuda().ref_single_scale(f_level, dptr(Im1), dptr(dm1), dptr(Im2), dptr(dm2), dptr(wI2), dptr(wD2),
                                         dptr(u), dptr(v), dptr(w), W, H, C, colorW, dptr(ddw), alpha, dptr(dsw),
                                         gamma, dptr(mag), dptr(regw), nOuter, nInner, nSOR, int(allowEarly))
        if rc != 0:
            raise RuntimeError("reference CUDA solver failed: cuda error %d" % rc)
        return u, v, w, wI2, wD2, None
    st = rf.Stats()
    rc = oracle().sfo_single_scale(int(fp64), f_level, dptr(Im1), dptr(dm1), dptr(Im2), dptr(dm2), dptr(wI2),
                                   dptr(wD2), dptr(u), dptr(v), dptr(w), W, H, C, colorW, dptr(ddw), alpha,
                                   dptr(dsw), gamma, dptr(mag), dptr(regw), nOuter, nInner, nSOR, int(allowEarly),
                                   ctypes.byref(params) if params is not None else None, ctypes.byref(st))
    if rc != 0:
        raise RuntimeError("oracle: %s" % oracle().sfo_last_error().decode())
    return u, v, w, wI2, wD2, st


def stereo_error1():
    """primesensor::stereoError(1) (src/primesensorUtils.cpp:53-56)."""
    return 1.0 / (1 / .00285 + 1.0)
