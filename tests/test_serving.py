"""The served form (continuous batching over camera streams) on a B200: every pair's result is
the same whether its stream is served alone or in a mix with other streams (bit-identical: the
kernels treat pairs independently and reduce in a fixed per-tile order), and cold-started served
pairs equal the plain solve."""
import os

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


# solve slots of a server (the library's default, or the RGBDFLOW_SERVER_SLOTS override)
SLOTS = int(os.environ.get("RGBDFLOW_SERVER_SLOTS", "4"))


def test_graphs_are_captured_when_a_stream_registers(ctx):
    """Registering a stream captures, on every solve slot, the graph of every batch the registered
    streams can form; the pairs that follow launch cached graphs only: the counters read no
    capture, no reallocation and no frame allocation, and one device step per pair."""
    seq = _streams()[0]
    srv = rf.Server(ctx, rf.benchmark_params(640), max_streams=4, max_batch=4, warm_start=False)
    fr = seq["frames"][0]
    srv.submit(0, 0, _cam(seq), fr["bgr"], fr["depth"])  # the stream's first frame registers it
    reg = srv.counters(reset=True)
    assert reg["graphs_built"] == SLOTS and reg["launches"] == 0 and reg["max_graph_build_ms"] > 0
    for k in range(1, 6):
        fr = seq["frames"][k % len(seq["frames"])]
        srv.submit(0, k, _cam(seq), fr["bgr"], fr["depth"])
        while srv.pending():
            for r in srv.step(wait=True):
                assert r[5] == 0
    c = srv.counters()
    assert c["graphs_built"] == 0 and c["arena_grows"] == 0 and c["frames_allocated"] == 0
    assert c["launches"] == 5
    assert c["max_submit_ms"] > 0 and c["max_launch_ms"] > 0 and c["max_retire_ms"] > 0
    srv.close()


def test_a_stream_registered_while_a_slot_runs_is_captured_before_its_next_launch(ctx):
    """A slot that is busy when a stream registers sizes its solve memory for that stream and
    captures its batches before it next launches (or at once, if it is idle by then): with a
    160x120 and a 320x240 stream, three batches per slot, and the mixed pairs that follow neither
    capture nor reallocate."""
    streams = _streams()
    srv = rf.Server(ctx, rf.benchmark_params(640), max_streams=4, max_batch=4, warm_start=False)

    def submit(s, k):
        fr = streams[s]["frames"][k]
        srv.submit(s, k, _cam(streams[s]), fr["bgr"], fr["depth"])

    def drain():
        while srv.pending():
            for r in srv.step(wait=True):
                assert r[5] == 0

    submit(0, 0)
    submit(0, 1)
    srv.step(wait=False)  # launches the first pair of stream 0 on a slot
    submit(1, 0)          # registers stream 1, most likely while that slot runs
    drain()
    start = srv.counters(reset=True)
    # per slot: the 160x120 batch when stream 0 registers; then its memory grows for the 320x240
    # stream (which drops its graphs) and it captures the three batches of the two streams
    assert start["graphs_built"] == SLOTS * (1 + 3) and start["arena_grows"] == SLOTS * 2
    for k in range(1, 5):
        submit(1, k)
        if k + 1 < 5:
            submit(0, k + 1)
        drain()
    c = srv.counters()
    assert c["graphs_built"] == 0 and c["arena_grows"] == 0 and c["launches"] == 4
    srv.close()
