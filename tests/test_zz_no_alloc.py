"""The allocation-free entry point (rgbdflow_scene_flow_noalloc) against the context entry point
that takes device pointers (rgbdflow_scene_flow_batch_async).

Both run the same plan and kernels, so the flows are expected to agree bit for bit; the test
allows 1e-6 (pixels for u and v, metres for w) per component.  Two calls in a row on one stream
check that the shared static workspace carries nothing from one call into the next; a third pair of
calls passes a warm start (the first solve's flow as est_flow) to both entry points.  This file is
collected last and also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import rgbdflow as rf
import synthetic as syn

TOL = 1e-6


def cam_of(p):
    c = p["cam"]
    return rf.CameraParams.make(p["W"], p["H"], c.f, c.cx, c.cy)


def device_pair(p, torch):
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return dict(W=p["W"], H=p["H"], cam=cam_of(p), bgr1=d(p["bgr1"]), depth1=d(p["depth1"]), bgr2=d(p["bgr2"]),
                depth2=d(p["depth2"]), out=torch.zeros((p["H"], p["W"], 3), dtype=torch.float32, device="cuda"))


def test_noalloc_rejects_oversized_pair():
    """A pair whose workspace exceeds the static array is refused before anything is enqueued."""
    lib = rf.load()
    buf = (ctypes.c_float * 16)()
    q = rf.RgbdFlowPair()
    q.W, q.H, q.cam = 640, 480, rf.CameraParams.make(640, 480, 525.0, 319.5, 239.5)
    q.bgr1 = q.bgr2 = ctypes.cast(buf, ctypes.c_void_p).value
    q.depth1_m = q.depth2_m = q.flow_out = ctypes.cast(buf, ctypes.c_void_p).value
    err = ctypes.create_string_buffer(256)
    rc = lib.rgbdflow_scene_flow_noalloc(ctypes.byref(q), ctypes.byref(rf.benchmark_params(640)), None, err, len(err))
    assert rc == -4  # RGBDFLOW_ERR_BUDGET
    assert b"static workspace" in err.value


@pytest.mark.gpu
def test_noalloc_matches_batch_async_two_calls(ctx):
    import torch
    prm = rf.benchmark_params(320)
    pairs = [device_pair(syn.make_config_pair("320x240", seed=s), torch) for s in (41, 42)]
    ref = [device_pair(syn.make_config_pair("320x240", seed=s), torch) for s in (41, 42)]
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        for p in ref:
            ctx.scene_flow_batch_device([p], prm, stream=st)
        st.synchronize()
        # two calls in a row on one stream: the second reuses the workspace the first just left
        rf.scene_flow_noalloc(pairs[0], prm, stream=st)
        rf.scene_flow_noalloc(pairs[1], prm, stream=st)
        st.synchronize()
    for p, r in zip(pairs, ref):
        a, b = p["out"].cpu().numpy(), r["out"].cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= TOL
        assert np.abs(a).max() > 0  # a real solve, not an untouched buffer


@pytest.mark.gpu
def test_noalloc_warm_start_matches_batch_async(ctx):
    """A warm start (est_flow, a device pointer) through both entry points."""
    import torch
    prm = rf.benchmark_params(320)
    p = syn.make_config_pair("320x240", seed=43)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        cold = device_pair(p, torch)
        ctx.scene_flow_batch_device([cold], prm, stream=st)
        st.synchronize()
        est = cold["out"].clone()
        a, b = device_pair(p, torch), device_pair(p, torch)
        a["est"] = est
        b["est"] = est
        ctx.scene_flow_batch_device([b], prm, stream=st)
        rf.scene_flow_noalloc(a, prm, stream=st)
        st.synchronize()
    x, y = a["out"].cpu().numpy(), b["out"].cpu().numpy()
    assert np.isfinite(x).all()
    assert np.abs(x - y).max() <= TOL
    assert np.abs(x - est.cpu().numpy()).max() > 0  # the warm-started solve moved the flow
