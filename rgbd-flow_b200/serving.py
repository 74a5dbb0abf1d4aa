"""Serving simulation: camera streams at a frame rate with Poisson (exponential inter-arrival)
jitter, driven through the continuous-batching server (rgbdflow.Server)."""
import time

import numpy as np

import synthetic as syn

STREAM_MIX = [("640x480", 5), ("320x240", 3)]  # 8 streams: 5 at 640x480, 3 at 320x240


def make_streams(n_unique=10, seed0=500, mix=STREAM_MIX):
    """Per stream: its camera and n_unique frames of a smooth rigid-trajectory sequence; longer
    sequences replay them forwards and backwards (consecutive frames always differ by one step)."""
    streams = []
    sid = 0
    for name, count in mix:
        cfg = dict(syn.CONFIGS[name])
        for _ in range(count):
            seq = syn.make_sequence(n_frames=n_unique, seed=seed0 + sid, **cfg)
            streams.append(seq)
            sid += 1
    return streams


def frame_index(t, n_unique):
    """Ping-pong replay: 0, 1, ..., n-1, n-2, ..., 1, 0, 1, ..."""
    period = 2 * (n_unique - 1)
    k = t % period
    return k if k < n_unique else period - k


def simulate(server, rf, streams, n_frames=300, fps=30.0, seed=0, time_scale=1.0, keep_stream=None, keep_n=0):
    """Submit n_frames per stream at `fps` (exponential inter-arrival times, mean 1/fps) and
    collect every result.  Returns dict(latencies_ms, pairs, wall_s, kept, host, span_s) where kept
    holds up to keep_n (frame index, flow) results of stream keep_stream, host the longest host
    times (ms) of one loop iteration (its sleep excluded), one submit call and one step call, and
    span_s the time of the last arrival."""
    rng = np.random.default_rng(seed)
    arrivals = []
    for s, seq in enumerate(streams):
        t = rng.exponential(1.0 / fps)
        for k in range(n_frames):
            arrivals.append((t * time_scale, s, k))
            t += rng.exponential(1.0 / fps)
    arrivals.sort()
    cams = [rf.CameraParams.make(seq["W"], seq["H"], seq["cam"].f, seq["cam"].cx, seq["cam"].cy) for seq in streams]
    lat, done, kept = [], 0, []
    host = dict(iter_ms=0.0, submit_ms=0.0, step_ms=0.0)
    t0 = time.perf_counter()
    i = 0
    # until every frame has arrived and every pair it formed has been returned (a stream that the
    # server already knows pairs its first frame here with its last frame of an earlier run)
    while i < len(arrivals) or server.pending() > 0:
        t_iter = time.perf_counter()
        now = t_iter - t0
        while i < len(arrivals) and arrivals[i][0] <= now:
            _, s, k = arrivals[i]
            seq = streams[s]
            fr = seq["frames"][frame_index(k, len(seq["frames"]))]
            t = time.perf_counter()
            server.submit(s, k, cams[s], fr["bgr"], fr["depth"])
            host["submit_ms"] = max(host["submit_ms"], 1e3 * (time.perf_counter() - t))
            i += 1
        wait = i >= len(arrivals)
        t = time.perf_counter()
        res = server.step(wait=wait)
        if not wait:
            host["step_ms"] = max(host["step_ms"], 1e3 * (time.perf_counter() - t))
        for (sid, rid, flow, ts, td, st) in res:
            if st != 0:
                raise RuntimeError("request failed: %d" % st)
            lat.append(1e3 * (td - ts))
            done += 1
            if sid == keep_stream and len(kept) < keep_n:
                kept.append((rid, flow))
        if not wait:
            host["iter_ms"] = max(host["iter_ms"], 1e3 * (time.perf_counter() - t_iter))
        if not res and i < len(arrivals):
            nxt = arrivals[i][0] - (time.perf_counter() - t0)
            if nxt > 0:
                time.sleep(min(nxt, 0.0005))
    wall = time.perf_counter() - t0
    return dict(latencies_ms=lat, pairs=done, wall_s=wall, kept=kept, host=host,
                span_s=arrivals[-1][0] if arrivals else 0.0)
