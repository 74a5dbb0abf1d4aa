"""Bounded device waits report a status the host reads, and the context stays usable.

The self-test (rgbdflow_debug_wait_timeout) runs one grid barrier that no other block reaches: the
wait runs out after its spin limit, the kernel records it in the context's status word and
returns, and the call reports RGBDFLOW_ERR_TIMEOUT.  Nothing faults or hangs: the barrier's wait
is bounded like every grid barrier of the solve.  A solve on the same context before and after
must give the same flows, and the status is reported once.
"""
import numpy as np
import pytest

import rgbdflow as rf
import synthetic as syn


def host_pair(p):
    c = p["cam"]
    return dict(W=p["W"], H=p["H"], cam=rf.CameraParams.make(p["W"], p["H"], c.f, c.cx, c.cy), bgr1=p["bgr1"],
                depth1=p["depth1"], bgr2=p["bgr2"], depth2=p["depth2"])


@pytest.mark.gpu
def test_wait_timeout_is_reported_and_the_context_stays_usable():
    ctx = rf.Context(0)
    try:
        prm = rf.benchmark_params(320)
        pair = host_pair(syn.make_config_pair("320x240", seed=7))
        before = ctx.scene_flow_batch([pair], prm, stats=False)[0]
        rc, sec = ctx.debug_wait_timeout()
        assert rc == -5, (rc, ctx.lib.rgbdflow_last_error(ctx.h))  # RGBDFLOW_ERR_TIMEOUT
        assert b"gave up" in ctx.lib.rgbdflow_last_error(ctx.h)
        assert 0.0 < sec < 30.0
        # reported once: synchronising afterwards succeeds, and so do solves
        ctx.synchronize()
        after = ctx.scene_flow_batch([pair], prm, stats=False)[0]
        assert np.array_equal(before, after)
        # the HPB path (its fill kernel has the same bounded barriers) also runs clean afterwards
        p2 = rf.benchmark_params(320)
        p2.regularization = rf.REG_HPB
        ctx.scene_flow_batch([pair], p2, stats=False)
        ctx.synchronize()
    finally:
        ctx.close()
