"""The served form (continuous batching over camera streams) on a B200: every pair's result is
the same whether its stream is served alone or in a mix with other streams (bit-identical: the
kernels treat pairs independently and reduce in a fixed per-tile order), and cold-started served
pairs equal the plain solve."""
import numpy as np
import pytest

import rgbdflow as rf
import synthetic as syn

pytestmark = pytest.mark.gpu


def _streams():
    out = []
    for i, name in enumerate(["160x120", "320x240", "160x120"]):
        cfg = dict(syn.CONFIGS[name])
        out.append(syn.make_sequence(n_frames=5, seed=40 + i, **cfg))
    return out


def _cam(seq):
    return rf.CameraParams.make(seq["W"], seq["H"], seq["cam"].f, seq["cam"].cx, seq["cam"].cy)


def _serve(ctx, streams, which, warm, interleave=True):
    srv = rf.Server(ctx, rf.benchmark_params(640), max_streams=4, max_batch=4, warm_start=warm,
                    warm_early_termination=warm)
    res = {}
    n = len(streams[0]["frames"])
    order = [(k, s) for k in range(n) for s in which] if interleave else [(k, s) for s in which for k in range(n)]
    for k, s in order:
        fr = streams[s]["frames"][k]
        srv.submit(s, k, _cam(streams[s]), fr["bgr"], fr["depth"])
        for (sid, rid, flow, ts, td, st) in srv.step(wait=False):
            assert st == 0
            res[(sid, rid)] = flow.copy()
    while srv.pending():
        for (sid, rid, flow, ts, td, st) in srv.step(wait=True):
            assert st == 0
            res[(sid, rid)] = flow.copy()
    srv.close()
    return res


@pytest.mark.parametrize("warm", [False, True])
def test_same_result_alone_and_in_the_mix(ctx, warm):
    streams = _streams()
    alone = _serve(ctx, streams, [0], warm)
    mixed = _serve(ctx, streams, [0, 1, 2], warm)
    assert len(alone) == 4 and len(mixed) == 12
    for k in range(1, 5):
        np.testing.assert_array_equal(alone[(0, k)], mixed[(0, k)])


def test_cold_served_pair_equals_plain_solve(ctx):
    streams = _streams()
    served = _serve(ctx, streams, [1, 2], warm=False, interleave=False)
    for s in (1, 2):
        seq = streams[s]
        for k in range(1, 5):
            f1, f2 = seq["frames"][k - 1], seq["frames"][k]
            plain = ctx.scene_flow_two_frames(_cam(seq), f1["bgr"], f1["depth"], f2["bgr"], f2["depth"],
                                              rf.benchmark_params(640), stats=False)
            np.testing.assert_array_equal(served[(s, k)], plain)


def test_admission_respects_the_hbm_budget(ctx):
    streams = _streams()
    srv = rf.Server(ctx, rf.benchmark_params(640), max_streams=4, max_batch=4, hbm_budget_bytes=1 << 20)
    fr = streams[1]["frames"][0]
    with pytest.raises(rf.RgbdFlowError) as e:
        srv.submit(1, 0, _cam(streams[1]), fr["bgr"], fr["depth"])  # a 320x240 frame + flow exceed 1 MB
    assert e.value.code == -4
    srv.close()
