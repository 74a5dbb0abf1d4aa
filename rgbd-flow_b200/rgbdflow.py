"""Python binding of librgbdflow.so (the C ABI declared in include/rgbdflow.h), via ctypes.

The library is the product: C++ host code plus hand-written sm_100a CUDA kernels.  This module
only marshals numpy arrays across the C ABI; it never computes flow itself and it raises if the
compiled library is missing (there is no CPU fallback).

Mirrors the reference's C++ entry points (paths inside eherbst/rgbd-flow):
  scene_flow_two_frames    runFlowTwoFramesSceneFlowExperiments   src/runFlowTwoFrames.cpp:109-121
  scene_flow_multiscale    OpticalFlow::sceneFlowMultiscale        src/sceneFlowMultiscale.cpp:30-201
  scene_flow_with_init     OpticalFlow::sceneFlowWithInit          src/sceneFlowWithInit.cpp:7-81
  scene_flow_single_scale  sceneFlowSingleScale                    src/sceneFlowSingleScaleJacobiCUDA.cu:660-969
Errors surface as RgbdFlowError carrying the library's status code and message (the reference
throws std::runtime_error from ASSERT_ALWAYS, include/rgbd_util/assert.h:57,106).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librgbdflow.so")

REG_ISOTROPIC, REG_LETOUZEY, REG_HPB = 0, 1, 2
STORE_FP32, STORE_FP16, STORE_BF16 = 0, 1, 2
# plane kinds of Context.debug_plane (RGBDFLOW_PLANE_* of include/rgbdflow.h)
(PLANE_PYRAMID, PLANE_FEATURES1, PLANE_FEATURES2, PLANE_DEPTH, PLANE_DEPTH_MAG, PLANE_REG, PLANE_FLOW, PLANE_SYSTEM,
 PLANE_FILL_ROUND, PLANE_HPB_DEPTH) = range(10)
COMPUTE_FP32, COMPUTE_FP64 = 0, 1
MAX_LEVELS, MAX_OUTER = 16, 64

OK = 0
ERR_NAMES = {-1: "INVALID_ARG", -2: "UNSUPPORTED", -3: "CUDA", -4: "BUDGET", -5: "TIMEOUT",
             -6: "NO_DEVICE", -7: "BUSY", -8: "INTERNAL", -9: "IO", -10: "FORMAT"}


class RgbdFlowError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERR_NAMES.get(code, "?"), code, msg))
        self.code = code


class CameraParams(ctypes.Structure):
    """rgbd::CameraParams (include/rgbd_util/CameraParams.h:17-28)."""
    _fields_ = [("xRes", ctypes.c_uint), ("yRes", ctypes.c_uint), ("centerX", ctypes.c_float),
                ("centerY", ctypes.c_float), ("focalLength", ctypes.c_float),
                ("stereoBaseline", ctypes.c_float), ("fovX", ctypes.c_float), ("fovY", ctypes.c_float)]

    @classmethod
    def make(cls, W, H, f, cx, cy):
        return cls(W, H, cx, cy, f, 0.072, 1.0472, 1.0472)


class Params(ctypes.Structure):
    _fields_ = [("regularization", ctypes.c_int), ("color_data_weight", ctypes.c_double),
                ("depth_vs_color_data_weight", ctypes.c_double), ("alpha", ctypes.c_double),
                ("gamma", ctypes.c_double), ("pyramid_ratio", ctypes.c_double), ("min_width", ctypes.c_int),
                ("n_outer", ctypes.c_int), ("n_inner", ctypes.c_int), ("n_sor", ctypes.c_int),
                ("depth_boundary_dist", ctypes.c_int), ("fill_holes", ctypes.c_int),
                ("fixed_schedule", ctypes.c_int), ("storage", ctypes.c_int), ("compute", ctypes.c_int),
                ("omega", ctypes.c_double), ("max_flow_step", ctypes.c_double), ("eps_d", ctypes.c_double),
                ("eps_z", ctypes.c_double), ("eps_s", ctypes.c_double), ("sor_tol", ctypes.c_double),
                ("sor_check_period", ctypes.c_int), ("outer_tol", ctypes.c_double),
                ("occ_margin", ctypes.c_double), ("occ_penalty", ctypes.c_double),
                ("max_depth_grad", ctypes.c_double), ("sweeps_per_launch", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("n_levels", ctypes.c_int), ("level_w", ctypes.c_int * MAX_LEVELS),
                ("level_h", ctypes.c_int * MAX_LEVELS), ("outer_iters", ctypes.c_int * MAX_LEVELS),
                ("sor_iters", (ctypes.c_int * MAX_OUTER) * MAX_LEVELS),
                ("outer_stat", (ctypes.c_float * MAX_OUTER) * MAX_LEVELS),
                ("sor_maxdiff", (ctypes.c_float * MAX_OUTER) * MAX_LEVELS),
                ("device_ms", ctypes.c_double)]

    def summary(self):
        """Executed schedule, finest level first: [(W, H, outer, [sor per outer])]."""
        out = []
        for k in range(self.n_levels):
            n = self.outer_iters[k]
            out.append((self.level_w[k], self.level_h[k], n, [self.sor_iters[k][o] for o in range(min(n, MAX_OUTER))]))
        return out


def default_params():
    """The reference defaults (sceneFlowParams() + setUpSceneFlowParams, runFlowTwoFrames.cpp:66-100),
    set without calling the library so it is usable on hosts without a GPU."""
    p = Params()
    p.regularization = REG_HPB
    p.color_data_weight = 1.0
    p.depth_vs_color_data_weight = 1.0
    p.alpha = 0.02
    p.gamma = 1e-5
    p.pyramid_ratio = 0.75
    p.min_width = 60
    p.n_outer, p.n_inner, p.n_sor = 50, 1, 10000
    p.depth_boundary_dist = 4
    p.fill_holes = 1
    p.fixed_schedule = 0
    p.storage = STORE_FP32
    p.compute = COMPUTE_FP32
    p.omega = 0.7
    p.max_flow_step = 0.3
    p.eps_d, p.eps_z, p.eps_s = 1e-6, 1e-10, 1e-6
    p.sor_tol = 1e-5
    p.sor_check_period = 25
    p.outer_tol = 4e-4
    p.occ_margin = 0.02
    p.occ_penalty = 0.01
    p.max_depth_grad = 0.04
    p.sweeps_per_launch = 0
    return p


def benchmark_params(W, **over):
    """The benchmark schedule: ISOTROPIC, ratio 0.5 with minWidth = W/16 for every pair (5 levels;
    min_width = -16), 10 outer, 1 inner, 30 SOR iterations, alpha 0.02, gamma 1e-5.  W is kept for
    call-site symmetry; the per-pair rule makes one parameter set serve a ragged batch."""
    p = default_params()
    p.regularization = REG_ISOTROPIC
    p.pyramid_ratio = 0.5
    p.min_width = -16
    p.n_outer, p.n_inner, p.n_sor = 10, 1, 30
    for k, v in over.items():
        setattr(p, k, v)
    return p


class KernelStat(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("launches", ctypes.c_int), ("ms", ctypes.c_double),
                ("bytes", ctypes.c_double)]


class RgbdFlowPair(ctypes.Structure):
    _fields_ = [("W", ctypes.c_int), ("H", ctypes.c_int), ("cam", CameraParams),
                ("bgr1", ctypes.c_void_p), ("depth1_m", ctypes.c_void_p), ("bgr2", ctypes.c_void_p),
                ("depth2_m", ctypes.c_void_p), ("est_flow", ctypes.c_void_p), ("flow_out", ctypes.c_void_p)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("max_streams", ctypes.c_int), ("max_batch", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_size_t), ("warm_start", ctypes.c_int),
                ("warm_early_termination", ctypes.c_int), ("params", Params)]


class Result(ctypes.Structure):
    _fields_ = [("stream_id", ctypes.c_int), ("request_id", ctypes.c_uint64), ("W", ctypes.c_int),
                ("H", ctypes.c_int), ("flow", ctypes.c_void_p), ("submit_time_s", ctypes.c_double),
                ("done_time_s", ctypes.c_double), ("status", ctypes.c_int)]


class Flow2dParams(ctypes.Structure):
    """rgbdflow_flow2d_params: the 2-D optical flow's parameters (the demo's flow type 1)."""
    _fields_ = [("alpha", ctypes.c_double), ("pyramid_ratio", ctypes.c_double), ("min_width", ctypes.c_int),
                ("n_outer", ctypes.c_int), ("n_inner", ctypes.c_int), ("n_sor", ctypes.c_int),
                ("sor_ring", ctypes.c_int)]


class ServerCounters(ctypes.Structure):
    _fields_ = [("frames_allocated", ctypes.c_uint64), ("graphs_built", ctypes.c_uint64),
                ("arena_grows", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("max_submit_ms", ctypes.c_double), ("max_launch_ms", ctypes.c_double),
                ("max_retire_ms", ctypes.c_double), ("max_graph_build_ms", ctypes.c_double)]


_lib = None

_P = ctypes.POINTER
_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double

# every symbol include/rgbdflow.h declares, with its ctypes signature
SIGNATURES = {
    "rgbdflow_params_default": (None, [_P(Params)]),
    "rgbdflow_abi_version": (_i, []),
    "rgbdflow_pyramid_levels": (_i, [_i, _i, _d, _i, _P(_i), _P(_i)]),
    "rgbdflow_batch_device_bytes": (_i, [_P(_i), _P(_i), _P(_i), _i, _P(Params), _P(ctypes.c_size_t)]),
    "rgbdflow_ctx_create": (_i, [_i, ctypes.c_size_t, _P(_vp)]),
    "rgbdflow_ctx_destroy": (_i, [_vp]),
    "rgbdflow_last_error": (ctypes.c_char_p, [_vp]),
    "rgbdflow_ctx_device_bytes": (ctypes.c_size_t, [_vp]),
    "rgbdflow_scene_flow_two_frames": (_i, [_vp, _P(CameraParams), _vp, _vp, _vp, _vp, _i, _i, _P(Params),
                                            _vp, _vp, _P(Stats)]),
    "rgbdflow_scene_flow_multiscale": (_i, [_vp, _P(CameraParams), _vp, _vp, _vp, _vp, _vp, _i, _i, _P(Params),
                                            _vp, _vp, _vp, _P(Stats)]),
    "rgbdflow_scene_flow_with_init": (_i, [_vp, _P(CameraParams), _vp, _vp, _vp, _vp, _vp, _i, _i, _P(Params),
                                           _vp, _vp, _vp, _P(Stats)]),
    "rgbdflow_scene_flow_single_scale": (_i, [_vp, _P(CameraParams)] + [_vp] * 9 + [_i, _i, _i, _d, _vp, _d, _vp, _d,
                                              _vp, _vp, _i, _i, _i, _i, _P(Params), _P(Stats)]),
    "rgbdflow_scene_flow_batch": (_i, [_vp, _P(RgbdFlowPair), _i, _P(Params), _P(Stats)]),
    "rgbdflow_scene_flow_batch_async": (_i, [_vp, _P(RgbdFlowPair), _i, _P(Params), _vp]),
    "rgbdflow_scene_flow_batch_submit": (_i, [_vp, _P(RgbdFlowPair), _i, _P(Params)]),
    "rgbdflow_ctx_synchronize": (_i, [_vp]),
    "rgbdflow_ctx_last_launch_count": (_i, [_vp]),
    "rgbdflow_profile": (_i, [_vp, _i]),
    "rgbdflow_profile_read": (_i, [_vp, _P(KernelStat), _i]),
    "rgbdflow_debug_read_plane": (_i, [_vp, _i, _i, _i, _i, _P(_d), ctypes.c_size_t, _P(_i), _P(_i)]),
    "rgbdflow_debug_wait_timeout": (_i, [_vp, _P(_d)]),
    "rgbdflow_autotune_describe": (_i, [_i, ctypes.c_char_p, ctypes.c_size_t]),
    "rgbdflow_server_create": (_i, [_vp, _P(ServerConfig), _P(_vp)]),
    "rgbdflow_server_destroy": (_i, [_vp]),
    "rgbdflow_server_submit": (_i, [_vp, _i, ctypes.c_uint64, _P(CameraParams), _vp, _vp, _i, _i, _vp]),
    "rgbdflow_server_step": (_i, [_vp, _i, _P(Result), _i, _P(_i)]),
    "rgbdflow_server_pending": (_i, [_vp]),
    "rgbdflow_server_counters_read": (_i, [_vp, _i, _P(ServerCounters)]),
    "rgbdflow_scene_flow_noalloc": (_i, [_P(RgbdFlowPair), _P(Params), _vp, ctypes.c_char_p, ctypes.c_size_t]),
    "rgbdflow_flow2d_params_default": (None, [_P(Flow2dParams)]),
    "rgbdflow_optical_flow_2d": (_i, [_vp, _vp, _vp, _i, _i, _P(Flow2dParams), _vp]),
    "rgbdflow_flo3_write": (_i, [ctypes.c_char_p, _vp, _i, _i, ctypes.c_char_p, ctypes.c_size_t]),
    "rgbdflow_flo3_read": (_i, [ctypes.c_char_p, _vp, ctypes.c_size_t, _P(_i), _P(_i), ctypes.c_char_p,
                                ctypes.c_size_t]),
    "rgbdflow_flo_write": (_i, [ctypes.c_char_p, _vp, _i, _i, ctypes.c_char_p, ctypes.c_size_t]),
    "rgbdflow_flo_read": (_i, [ctypes.c_char_p, _vp, ctypes.c_size_t, _P(_i), _P(_i), ctypes.c_char_p,
                               ctypes.c_size_t]),
}


def load():
    """Load librgbdflow.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RgbdFlowError(-6, "librgbdflow.so not built at %s (run __graft_entry__.build())" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def pyramid_levels(W, H, ratio, min_width):
    """[(w, h)] of the solve's pyramid, finest first (host-only)."""
    lib = load()
    w = (ctypes.c_int * MAX_LEVELS)()
    h = (ctypes.c_int * MAX_LEVELS)()
    n = lib.rgbdflow_pyramid_levels(W, H, ratio, min_width, w, h)
    if n < 0:
        raise RgbdFlowError(n, "rgbdflow_pyramid_levels failed")
    return [(w[i], h[i]) for i in range(n)]


def batch_device_bytes(sizes, params, warm=None):
    """Device bytes a batch of (W, H) sizes needs (host-only)."""
    lib = load()
    n = len(sizes)
    Ws = (ctypes.c_int * n)(*[s[0] for s in sizes])
    Hs = (ctypes.c_int * n)(*[s[1] for s in sizes])
    wm = (ctypes.c_int * n)(*([int(bool(x)) for x in warm] if warm else [0] * n))
    out = ctypes.c_size_t()
    rc = lib.rgbdflow_batch_device_bytes(Ws, Hs, wm, n, ctypes.byref(params), ctypes.byref(out))
    if rc != OK:
        raise RgbdFlowError(rc, "rgbdflow_batch_device_bytes failed")
    return out.value


def flow2d_params(**over):
    """rgbdflow_flow2d_params_default (the demo's flow type 1: alpha 0.02, ratio 0.75, minWidth 20,
    10 outer, 1 inner, 400 SOR iterations) with the given fields replaced.  Host-only."""
    p = Flow2dParams()
    load().rgbdflow_flow2d_params_default(ctypes.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _write_flow_file(fn, path, flow, C):
    flow = np.ascontiguousarray(flow, dtype=np.float32)
    if flow.ndim != 3 or flow.shape[2] != C:
        raise RgbdFlowError(-1, "flow must be (H, W, %d)" % C)
    err = ctypes.create_string_buffer(512)
    rc = fn(os.fsencode(path), _ptr(flow), flow.shape[1], flow.shape[0], err, len(err))
    if rc != OK:
        raise RgbdFlowError(rc, err.value.decode())


def _read_flow_file(fn, path, C):
    err = ctypes.create_string_buffer(512)
    W, H = ctypes.c_int(), ctypes.c_int()
    rc = fn(os.fsencode(path), None, 0, ctypes.byref(W), ctypes.byref(H), err, len(err))
    if rc != OK:
        raise RgbdFlowError(rc, err.value.decode())
    flow = np.empty((H.value, W.value, C), np.float32)
    rc = fn(os.fsencode(path), _ptr(flow), flow.size, ctypes.byref(W), ctypes.byref(H), err, len(err))
    if rc != OK:
        raise RgbdFlowError(rc, err.value.decode())
    return flow


def write_flo3(path, flow):
    """Write an (H, W, 3) float32 flow (u px, v px, w m) as a .flo3 file (rgbdflow_flo3_write;
    writeSceneFlow, src/sceneFlowIO.cpp:49-61).  Host-only."""
    _write_flow_file(load().rgbdflow_flo3_write, path, flow, 3)


def read_flo3(path):
    """Read a .flo3 file into an (H, W, 3) float32 array (rgbdflow_flo3_read; readSceneFlow,
    src/sceneFlowIO.cpp:23-44).  Host-only."""
    return _read_flow_file(load().rgbdflow_flo3_read, path, 3)


def write_flo(path, flow):
    """Write an (H, W, 2) float32 2-D flow as a Middlebury .flo file (rgbdflow_flo_write; writeFlow,
    src/middleburyFlowIO.cpp:50-65).  Host-only."""
    _write_flow_file(load().rgbdflow_flo_write, path, flow, 2)


def read_flo(path):
    """Read a Middlebury .flo file into an (H, W, 2) float32 array (rgbdflow_flo_read; readFlow,
    src/middleburyFlowIO.cpp:22-44).  Host-only."""
    return _read_flow_file(load().rgbdflow_flo_read, path, 2)


def autotune_describe(device=0):
    """The SOR configurations the autotuner chose on `device` (rgbdflow_autotune_describe)."""
    lib = load()
    n = lib.rgbdflow_autotune_describe(device, None, 0)
    buf = ctypes.create_string_buffer(max(n, 0) + 1)
    lib.rgbdflow_autotune_describe(device, buf, len(buf))
    return buf.value.decode()


def scene_flow_noalloc(pair, params, stream=None):
    """Allocation-free solve of one pair of torch CUDA tensors (keys as in
    Context.scene_flow_batch_device) in the library's static workspace, enqueued on `stream`
    (a torch.cuda.Stream, default: torch's current stream); returns without waiting."""
    import torch
    lib = load()
    arr = RgbdFlowPair()
    arr.W, arr.H, arr.cam = pair["W"], pair["H"], pair["cam"]
    arr.bgr1, arr.depth1_m = pair["bgr1"].data_ptr(), pair["depth1"].data_ptr()
    arr.bgr2, arr.depth2_m = pair["bgr2"].data_ptr(), pair["depth2"].data_ptr()
    arr.est_flow = pair["est"].data_ptr() if pair.get("est") is not None else None
    arr.flow_out = pair["out"].data_ptr()
    s = stream if stream is not None else torch.cuda.current_stream()
    err = ctypes.create_string_buffer(512)
    rc = lib.rgbdflow_scene_flow_noalloc(ctypes.byref(arr), ctypes.byref(params), ctypes.c_void_p(s.cuda_stream),
                                         err, len(err))
    if rc != OK:
        raise RgbdFlowError(rc, err.value.decode())


class Context:
    """One device context (stream, workspaces, cached graphs).  Not shared across threads."""

    def __init__(self, device=0, hbm_budget_bytes=0):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.rgbdflow_ctx_create(device, hbm_budget_bytes, ctypes.byref(h))
        if rc != OK:
            raise RgbdFlowError(rc, "rgbdflow_ctx_create failed")
        self.h = h

    def close(self):
        if self.h:
            self.lib.rgbdflow_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != OK:
            msg = self.lib.rgbdflow_last_error(self.h)
            raise RgbdFlowError(rc, msg.decode() if msg else "")

    def device_bytes(self):
        return self.lib.rgbdflow_ctx_device_bytes(self.h)

    def optical_flow_2d(self, bgr1, bgr2, params=None):
        """2-D optical flow (the reference demo's flow type 1; rgbdflow_optical_flow_2d) of two
        (H, W, 3) uint8 BGR frames: (H, W, 2) float32 (u, v in pixels)."""
        b1, b2 = _c(bgr1, np.uint8), _c(bgr2, np.uint8)
        H, W = b1.shape[:2]
        if b2.shape != b1.shape or b1.ndim != 3 or b1.shape[2] != 3:
            raise RgbdFlowError(-1, "frames must be two (H, W, 3) uint8 images of one size")
        out = np.empty((H, W, 2), np.float32)
        p = params if params is not None else flow2d_params()
        self._check(self.lib.rgbdflow_optical_flow_2d(self.h, _ptr(b1), _ptr(b2), W, H, ctypes.byref(p), _ptr(out)))
        return out

    def scene_flow_two_frames(self, cam, bgr1, depth1, bgr2, depth2, params, est_flow=None, stats=True):
        bgr1, bgr2 = _c(bgr1, np.uint8), _c(bgr2, np.uint8)
        depth1, depth2 = _c(depth1, np.float32), _c(depth2, np.float32)
        H, W = depth1.shape
        out = np.zeros((H, W, 3), np.float32)
        est = _c(est_flow, np.float32) if est_flow is not None else None
        st = Stats() if stats else None
        rc = self.lib.rgbdflow_scene_flow_two_frames(self.h, ctypes.byref(cam), _ptr(bgr1), _ptr(depth1), _ptr(bgr2),
                                                     _ptr(depth2), W, H, ctypes.byref(params), _ptr(est), _ptr(out),
                                                     ctypes.byref(st) if st is not None else None)
        self._check(rc)
        return (out, st) if stats else out

    def _dimage_call(self, fn, cam, Im1, dm1, Im2, dm2, sigma1, params, u=None, v=None, w=None):
        Im1, Im2 = _c(Im1, np.float64), _c(Im2, np.float64)
        dm1, dm2 = _c(dm1, np.float64), _c(dm2, np.float64)
        sigma1 = _c(sigma1, np.float32)
        H, W = dm1.shape
        u = np.zeros((H, W)) if u is None else _c(u, np.float64).copy()
        v = np.zeros((H, W)) if v is None else _c(v, np.float64).copy()
        w = np.zeros((H, W)) if w is None else _c(w, np.float64).copy()
        st = Stats()
        rc = fn(self.h, ctypes.byref(cam), _ptr(Im1), _ptr(dm1), _ptr(Im2), _ptr(dm2), _ptr(sigma1), W, H,
                ctypes.byref(params), _ptr(u), _ptr(v), _ptr(w), ctypes.byref(st))
        self._check(rc)
        return u, v, w, st

    def scene_flow_multiscale(self, cam, Im1, dm1, Im2, dm2, sigma1, params):
        """OpticalFlow::sceneFlowMultiscale on DImage-style FP64 buffers; returns (u, v, w, stats)."""
        return self._dimage_call(self.lib.rgbdflow_scene_flow_multiscale, cam, Im1, dm1, Im2, dm2, sigma1, params)

    def scene_flow_with_init(self, cam, Im1, dm1, Im2, dm2, sigma1, params, u, v, w):
        """OpticalFlow::sceneFlowWithInit: one full-resolution level from the estimate (u, v, w)."""
        return self._dimage_call(self.lib.rgbdflow_scene_flow_with_init, cam, Im1, dm1, Im2, dm2, sigma1, params,
                                 u, v, w)

    def scene_flow_single_scale(self, cam, Im1, dm1, Im2, dm2, warpIm2, warpDm2, u, v, w, colorW, ddw, alpha, dsw,
                                gamma, mag, regw, nOuter, nInner, nSOR, allowEarly, params=None):
        Im1, Im2 = _c(Im1, np.float64), _c(Im2, np.float64)
        dm1, dm2 = _c(dm1, np.float64), _c(dm2, np.float64)
        warpIm2, warpDm2 = _c(warpIm2, np.float64).copy(), _c(warpDm2, np.float64).copy()
        u, v, w = _c(u, np.float64).copy(), _c(v, np.float64).copy(), _c(w, np.float64).copy()
        ddw, dsw, mag, regw = (_c(x, np.float64) for x in (ddw, dsw, mag, regw))
        H, W, C = Im1.shape
        st = Stats()
        rc = self.lib.rgbdflow_scene_flow_single_scale(
            self.h, ctypes.byref(cam), _ptr(Im1), _ptr(dm1), _ptr(Im2), _ptr(dm2), _ptr(warpIm2), _ptr(warpDm2),
            _ptr(u), _ptr(v), _ptr(w), W, H, C, colorW, _ptr(ddw), alpha, _ptr(dsw), gamma, _ptr(mag), _ptr(regw),
            nOuter, nInner, nSOR, int(allowEarly), ctypes.byref(params) if params is not None else None,
            ctypes.byref(st))
        self._check(rc)
        return u, v, w, warpIm2, warpDm2, st

    def last_launch_count(self):
        return self.lib.rgbdflow_ctx_last_launch_count(self.h)

    def synchronize(self):
        self._check(self.lib.rgbdflow_ctx_synchronize(self.h))

    def profile(self, enable):
        self._check(self.lib.rgbdflow_profile(self.h, int(enable)))

    def profile_read(self):
        """{kernel class: (launches, ms, algorithmic bytes)} accumulated while profiling."""
        buf = (KernelStat * 32)()
        n = self.lib.rgbdflow_profile_read(self.h, buf, 32)
        return {buf[i].name.decode(): (buf[i].launches, buf[i].ms, buf[i].bytes) for i in range(min(n, 32))}

    def debug_plane(self, pair, level, kind, index=0):
        """Plane (kind, index) of pair `pair`, pyramid level `level` of the last solve, as an (H, W)
        float64 array (rgbdflow_debug_read_plane; kind is one of the PLANE_* constants)."""
        w, h = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.lib.rgbdflow_debug_read_plane(self.h, pair, level, kind, index, None, 0, ctypes.byref(w),
                                                       ctypes.byref(h)))
        out = np.zeros((h.value, w.value), np.float64)
        self._check(self.lib.rgbdflow_debug_read_plane(self.h, pair, level, kind, index,
                                                       out.ctypes.data_as(_P(_d)), out.size, None, None))
        return out

    def debug_wait_timeout(self):
        """Runs the bounded-wait self-test (rgbdflow_debug_wait_timeout): (status code, seconds the
        wait took).  RGBDFLOW_ERR_TIMEOUT is the expected code."""
        sec = ctypes.c_double(0)
        rc = self.lib.rgbdflow_debug_wait_timeout(self.h, ctypes.byref(sec))
        return rc, sec.value

    def scene_flow_batch_device(self, pairs, params, stream=None):
        """Device-pointer batch: pairs hold torch CUDA tensors (bgr1/bgr2 uint8 HxWx3, depth1/depth2
        float32 HxW, out float32 HxWx3, optional est float32 HxWx3).  Enqueued on `stream` (a
        torch.cuda.Stream, default: torch's current stream); returns without waiting."""
        import torch
        arr = (RgbdFlowPair * len(pairs))()
        for i, p in enumerate(pairs):
            arr[i].W, arr[i].H, arr[i].cam = p["W"], p["H"], p["cam"]
            arr[i].bgr1, arr[i].depth1_m = p["bgr1"].data_ptr(), p["depth1"].data_ptr()
            arr[i].bgr2, arr[i].depth2_m = p["bgr2"].data_ptr(), p["depth2"].data_ptr()
            arr[i].est_flow = p["est"].data_ptr() if p.get("est") is not None else None
            arr[i].flow_out = p["out"].data_ptr()
        s = stream if stream is not None else torch.cuda.current_stream()
        handle = s.cuda_stream
        if handle == 0:
            handle = 1  # torch's default stream is the legacy stream: cudaStreamLegacy, not NULL (NULL = the context's stream)
        rc = self.lib.rgbdflow_scene_flow_batch_async(self.h, arr, len(pairs), ctypes.byref(params),
                                                      ctypes.c_void_p(handle))
        self._check(rc)

    def scene_flow_batch(self, pairs, params, stats=True, outs=None):
        """pairs: list of dicts with W, H, cam (CameraParams), bgr1, depth1, bgr2, depth2[, est_flow].
        outs: optional preallocated (H,W,3) float32 arrays (page-locked ones are filled by DMA).
        Returns the list of (H,W,3) float32 flows (and Stats list)."""
        keep = []
        arr = (RgbdFlowPair * len(pairs))()
        given = outs
        outs = []
        for i, p in enumerate(pairs):
            b1, b2 = _c(p["bgr1"], np.uint8), _c(p["bgr2"], np.uint8)
            d1, d2 = _c(p["depth1"], np.float32), _c(p["depth2"], np.float32)
            est = _c(p["est_flow"], np.float32) if p.get("est_flow") is not None else None
            out = given[i] if given is not None else np.zeros((p["H"], p["W"], 3), np.float32)
            keep += [b1, b2, d1, d2, est, out]
            outs.append(out)
            arr[i].W, arr[i].H, arr[i].cam = p["W"], p["H"], p["cam"]
            arr[i].bgr1, arr[i].depth1_m = b1.ctypes.data, d1.ctypes.data
            arr[i].bgr2, arr[i].depth2_m = b2.ctypes.data, d2.ctypes.data
            arr[i].est_flow = est.ctypes.data if est is not None else None
            arr[i].flow_out = out.ctypes.data
        st = (Stats * len(pairs))() if stats else None
        rc = self.lib.rgbdflow_scene_flow_batch(self.h, arr, len(pairs), ctypes.byref(params), st)
        self._check(rc)
        return (outs, list(st)) if stats else outs

    def scene_flow_batch_submit(self, pairs, params, outs):
        """Host-buffer batch that returns once enqueued (rgbdflow_scene_flow_batch_submit).  outs:
        page-locked (H,W,3) float32 arrays the flows are DMA'd into; the input arrays and outs must
        stay alive and unchanged until synchronize().  Returns outs."""
        keep = []
        arr = (RgbdFlowPair * len(pairs))()
        for i, p in enumerate(pairs):
            b1, b2 = _c(p["bgr1"], np.uint8), _c(p["bgr2"], np.uint8)
            d1, d2 = _c(p["depth1"], np.float32), _c(p["depth2"], np.float32)
            est = _c(p["est_flow"], np.float32) if p.get("est_flow") is not None else None
            keep += [b1, b2, d1, d2, est]
            arr[i].W, arr[i].H, arr[i].cam = p["W"], p["H"], p["cam"]
            arr[i].bgr1, arr[i].depth1_m = b1.ctypes.data, d1.ctypes.data
            arr[i].bgr2, arr[i].depth2_m = b2.ctypes.data, d2.ctypes.data
            arr[i].est_flow = est.ctypes.data if est is not None else None
            arr[i].flow_out = outs[i].ctypes.data
        rc = self.lib.rgbdflow_scene_flow_batch_submit(self.h, arr, len(pairs), ctypes.byref(params))
        self._check(rc)
        self._submitted = keep  # the staged / DMA'd inputs stay referenced until the next call
        return outs


class Server:
    """Continuous-batching server over camera streams (rgbdflow_server_*).  A frame submitted on a
    stream forms a pair with that stream's previous frame; its flow (previous -> this frame) lands
    in an array owned by this object until the request completes."""

    def __init__(self, ctx, params, max_streams=8, max_batch=8, hbm_budget_bytes=20 << 30, warm_start=True,
                 warm_early_termination=False):
        self.ctx = ctx
        self.lib = ctx.lib
        cfg = ServerConfig()
        cfg.max_streams, cfg.max_batch = max_streams, max_batch
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.warm_start = int(bool(warm_start))
        cfg.warm_early_termination = int(bool(warm_early_termination))
        cfg.params = params
        h = ctypes.c_void_p()
        rc = self.lib.rgbdflow_server_create(ctx.h, ctypes.byref(cfg), ctypes.byref(h))
        ctx._check(rc)
        self.h = h
        self._live = {}  # (stream, id) -> (out array, input arrays kept alive until the upload is staged)
        self._res = (Result * 64)()

    def submit(self, stream, req_id, cam, bgr, depth):
        bgr = _c(bgr, np.uint8)
        depth = _c(depth, np.float32)
        H, W = depth.shape
        out = np.empty((H, W, 3), np.float32)
        rc = self.lib.rgbdflow_server_submit(self.h, stream, req_id, ctypes.byref(cam), _ptr(bgr), _ptr(depth), W, H,
                                             _ptr(out))
        self.ctx._check(rc)
        self._live[(stream, req_id)] = out
        return out

    def step(self, wait=False):
        """Advance the device; returns [(stream, id, flow, submit_s, done_s, status)] of completed pairs."""
        n = ctypes.c_int()
        rc = self.lib.rgbdflow_server_step(self.h, int(wait), self._res, 64, ctypes.byref(n))
        self.ctx._check(rc)
        out = []
        for i in range(n.value):
            r = self._res[i]
            flow = self._live.pop((r.stream_id, r.request_id), None)
            out.append((r.stream_id, r.request_id, flow, r.submit_time_s, r.done_time_s, r.status))
        return out

    def pending(self):
        return self.lib.rgbdflow_server_pending(self.h)

    def counters(self, reset=False):
        """Host-side events that add to served latency (rgbdflow_server_counters_read): frame
        buffers allocated beyond the stock, graphs captured, arena reallocations, device steps, and
        the longest host time of a submit, a step launch, a step retirement and a graph capture +
        instantiation (ms)."""
        k = ServerCounters()
        self.ctx._check(self.lib.rgbdflow_server_counters_read(self.h, int(bool(reset)), ctypes.byref(k)))
        return {name: getattr(k, name) for name, _ in ServerCounters._fields_}

    def close(self):
        if self.h:
            self.lib.rgbdflow_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
