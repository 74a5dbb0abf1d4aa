#!/usr/bin/env python
"""Benchmark of the B200 scene-flow solve: 640x480 pairs/s.

A step is one batched solve of B synthetic 640x480 RGB-D pairs (B = 16 by default) with the
reference's schedule restated for the benchmark: ISOTROPIC regularisation, pyramid ratio 0.5 with
minWidth = W/16 (5 levels), 10 outer warps, 1 inner, 30 red-black SOR iterations, the reference's
convergence breaks and outer early termination on.  Every pair is an independent unit, so N GPUs
run N replicas (weak scaling, no collective on the data path).

  value      pairs/s with inputs resident in HBM (device-pointer API), two batches in flight on two
             contexts / streams, timed with CUDA events across the streams, max over ranks; the
             batch's solve memory (~1.5 GB) is far above L2.  `one_batch_in_flight` beside it.
  e2e        pairs/s through the host-buffer C ABI (rgbdflow_scene_flow_batch_submit on two
             contexts in rotation), every step's host->device inputs and device->host flows inside
             the timed region
  plain      one pair per call (the drop-in solve): pairs/s and p50 / p99 latency
  roofline   the dominant kernel (red-black SOR) from a profiled pass of the same workload
  cpu_baseline  the CPU restatement of the reference (oracle, all host threads) on one pair

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rgbd-flow_b200"))

import synthetic as syn  # noqa: E402

METRIC = "640×480 pairs/s & p99 latency, served+batched vs plain GPU at matched 3-D EPE"
W, H = 640, 480


def peaks():
    try:
        m = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic():
    """DRAM bytes of a level-0 strip-SOR launch per pair, from the committed ncu summary
    (profiles/sor_traffic.json), if present."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "sor_traffic.json")))
        return d
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.p = None
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="rgbdflow_clocks_rank%d_" % index, suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        self.p.wait()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def compact(x):
    """Floats rounded to 5 significant digits (keeps the one-line record short)."""
    if isinstance(x, float):
        return float("%.5g" % x)
    if isinstance(x, dict):
        return {k: compact(v) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [compact(v) for v in x]
    return x


def make_pairs(n, seed0):
    out = []
    for i in range(n):
        p = syn.make_config_pair("640x480", seed=seed0 + i)
        out.append(p)
    return out


def cam_of(rf, p):
    c = p["cam"]
    return rf.CameraParams.make(p["W"], p["H"], c.f, c.cx, c.cy)


def oracle_pairs_per_s(pairs, steps):
    """The CPU restatement on the host cores: one 640x480 pair per step."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    import rgbdflow as rf
    ob.build_oracle()
    threads = ob.oracle().sfo_set_threads(0)
    prm = rf.benchmark_params(W)
    outs, ts = [], []
    for s in range(steps):
        p = pairs[s % len(pairs)]
        t = time.perf_counter()
        f, _ = ob.two_frames(cam_of(rf, p), p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
        ts.append(time.perf_counter() - t)
        outs.append(f)
    return steps / sum(ts), threads, outs, ts


def device_pair(rf, torch, p):
    return dict(W=p["W"], H=p["H"], cam=cam_of(rf, p),
                bgr1=torch.from_numpy(p["bgr1"]).cuda(), bgr2=torch.from_numpy(p["bgr2"]).cuda(),
                depth1=torch.from_numpy(p["depth1"]).cuda(), depth2=torch.from_numpy(p["depth2"]).cuda(),
                out=torch.empty((p["H"], p["W"], 3), dtype=torch.float32, device="cuda"))


def run_ncu_case(n_pairs, rf, torch, storage="fp32", reg="isotropic"):
    """One batched solve of n_pairs 640x480 pairs through the device-pointer API, graphs off, with
    the feature / depth pyramids stored as `storage` and the given regularisation."""
    ctx = rf.Context(0)
    dev = [device_pair(rf, torch, p) for p in make_pairs(n_pairs, 0)]
    prm = rf.benchmark_params(W)
    prm.storage = {"fp32": rf.STORE_FP32, "fp16": rf.STORE_FP16, "bf16": rf.STORE_BF16}[storage]
    prm.regularization = {"isotropic": rf.REG_ISOTROPIC, "letouzey": rf.REG_LETOUZEY, "hpb": rf.REG_HPB}[reg]
    ctx.scene_flow_batch_device(dev, prm)
    torch.cuda.synchronize()
    ctx.close()


def run_served(ctx, rf, serving, streams, prm, args, warm):
    """Camera streams through the server: pairs/s, latency percentiles and the 3-D EPE of the
    served flows against the plain solve of the same pairs (stream 0, a few kept results)."""
    srv = rf.Server(ctx, prm, max_streams=len(streams), max_batch=len(streams), hbm_budget_bytes=20 << 30,
                    warm_start=warm, warm_early_termination=warm)
    # warm-up: the slots' graphs for the batch mixes that recur (about a second of traffic)
    serving.simulate(srv, rf, streams, n_frames=4 * args.serve_unique, fps=30.0, seed=1)
    srv.counters(reset=True)
    r = serving.simulate(srv, rf, streams, n_frames=args.serve_frames, fps=30.0, seed=2, keep_stream=0, keep_n=16)
    counters = srv.counters()
    lat = np.array(r["latencies_ms"])
    sat = serving.simulate(srv, rf, streams, n_frames=args.serve_unique * 3, fps=30.0, seed=3, time_scale=0.0)
    srv.close()
    seq = streams[0]
    epes, gt_served, gt_plain = [], [], []
    for rid, flow in r["kept"]:
        if rid == 0:
            continue  # its first frame is the last frame of the warm-up run, not frame_index(-1)
        n = len(seq["frames"])
        i1, i2 = serving.frame_index(rid - 1, n), serving.frame_index(rid, n)
        f1, f2 = seq["frames"][i1], seq["frames"][i2]
        camp = rf.CameraParams.make(seq["W"], seq["H"], seq["cam"].f, seq["cam"].cx, seq["cam"].cy)
        plain_f = ctx.scene_flow_two_frames(camp, f1["bgr"], f1["depth"], f2["bgr"], f2["depth"], prm, stats=False)
        z = np.where(f1["depth"] > 0, f1["depth"], 2.0).astype(np.float64)
        epes.append(syn.epe3d(flow, plain_f, z, seq["cam"], f1["depth"] > 0)[0])
        if i2 == i1 + 1:  # a forward pair: the sequence's analytic motion is its ground truth
            m = f1["depth"] > 0
            gt_served.append(syn.epe3d(flow, f1["gt_next"], f1["z_true"], seq["cam"], m)[0])
            gt_plain.append(syn.epe3d(plain_f, f1["gt_next"], f1["z_true"], seq["cam"], m)[0])
    how = ("warm starts from the stream's previous flow (full-resolution level, early termination allowed)"
           if warm else "cold: the full coarse-to-fine solve per pair (flows equal the plain call's)")
    return {"streams": "5 x 640x480 + 3 x 320x240 at 30 fps, Poisson arrivals; " + how,
            "pairs": r["pairs"], "pairs_per_s": r["pairs"] / r["wall_s"],
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()),
            "saturated_pairs_per_s": sat["pairs"] / sat["wall_s"],
            "epe_vs_plain_mm": 1e3 * float(np.mean(epes)) if epes else None,
            "epe_vs_ground_truth_mm": ({"served": 1e3 * float(np.mean(gt_served)), "plain": 1e3 * float(np.mean(gt_plain)),
                                        "pairs": len(gt_served)} if gt_served else None),
            "hbm_budget_gb": 20,
            # what the timed run spent on the host outside the solve: server counters (allocations,
            # graph captures, longest calls) and the request loop's longest iteration and calls
            "host": {"server": counters, "loop_ms": r["host"]}}


def run_served_sweep(ctx, rf, serving, base, prm, warm, points, seconds=2.0, max_batch=8):
    """Served capacity: camera streams (the 8 base streams replayed as more independent streams) at
    30 fps with Poisson arrivals, more streams per point.  Per point: the arrival rate actually
    drawn (pairs / time of the last arrival), the achieved pairs/s (pairs / wall time, which adds
    the last results' latency) and p50 / p99 latency; the result is the highest arrival rate served
    with p99 under 33 ms.  A server admits up to max_batch pairs a device step (one pair per stream
    in flight).  Stops after the first point whose p99 reaches 33 ms or whose results fall behind
    the arrivals by more than 20 %."""
    pts, best = [], None
    for n_streams, fps in points:
        streams = [base[i % len(base)] for i in range(n_streams)]
        srv = rf.Server(ctx, prm, max_streams=n_streams, max_batch=min(n_streams, max_batch),
                        hbm_budget_bytes=20 << 30, warm_start=warm, warm_early_termination=warm)
        serving.simulate(srv, rf, streams, n_frames=12, fps=float(fps), seed=11)  # graphs, memory
        r = serving.simulate(srv, rf, streams, n_frames=max(12, int(seconds * fps)), fps=float(fps),
                             seed=100 + n_streams)
        srv.close()
        lat = np.array(r["latencies_ms"])
        pt = {"streams": n_streams, "fps": fps, "arrivals_per_s": r["pairs"] / max(r["span_s"], 1e-9),
              "pairs_per_s": r["pairs"] / r["wall_s"], "wall_s": r["wall_s"], "span_s": r["span_s"],
              "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99))}
        pts.append(pt)
        if pt["p99_ms"] < 33.0 and (best is None or pt["arrivals_per_s"] > best["arrivals_per_s"]):
            best = pt
        if pt["p99_ms"] >= 33.0 or pt["pairs_per_s"] < 0.8 * pt["arrivals_per_s"]:
            break
    return {"mode": "warm" if warm else "cold", "max_batch": max_batch, "points": pts,
            "max_pairs_per_s_p99_under_33ms": best["arrivals_per_s"] if best else None}


MIX = [(160, 120, 24), (320, 240, 24), (640, 480, 16)]
# batches in flight (contexts / streams) of the value and e2e measurements: with three the
# device-resident value read 758 against 743 pairs/s, but e2e fell from 682 to 652
LANES = 2


def run_mixed(ctx, rf, torch, stream, prm, args, rank):
    """64 uneven pairs per step, device-resident, CUDA events on the launching stream."""
    dev = []
    for (w, h, n) in MIX:
        name = "%dx%d" % (w, h)
        for i in range(n):
            dev.append(device_pair(rf, torch, syn.make_config_pair(name, seed=3000 + 97 * rank + 1000 * w + i)))
    for _ in range(args.warmup):
        ctx.scene_flow_batch_device(dev, prm)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 10))
    e0.record(stream)
    for _ in range(steps):
        ctx.scene_flow_batch_device(dev, prm)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    px = sum(w * h * n for (w, h, n) in MIX)
    return {"pairs": len(dev), "mix": "24 x 160x120 + 24 x 320x240 + 16 x 640x480", "ms_per_step": ms,
            "pairs_per_s": 1e3 * len(dev) / ms, "equiv_640x480_pairs_per_s": 1e3 * px / (640 * 480) / ms,
            "launches_per_step": ctx.last_launch_count()}


def run_precision(ctx, rf, torch, stream, dev, pairs, args):
    """FP16 / BF16 pyramid storage against the FP32 and FP64 device solves of the same pairs."""
    n = min(4, len(dev))
    host = [dict(W=p["W"], H=p["H"], cam=cam_of(rf, p), bgr1=p["bgr1"], depth1=p["depth1"], bgr2=p["bgr2"],
                 depth2=p["depth2"]) for p in pairs[:n]]

    def epes(fl, ref):
        return [syn.epe3d(a, b, p["z1_true"], p["cam"], p["depth1"] > 0) for a, b, p in zip(fl, ref, pairs)]

    p64 = rf.benchmark_params(W)
    p64.compute = rf.COMPUTE_FP64
    f64 = ctx.scene_flow_batch(host, p64, stats=False)
    p32 = rf.benchmark_params(W)
    f32 = ctx.scene_flow_batch(host, p32, stats=False)
    dev = [dict(d, out=torch.empty_like(d["out"])) for d in dev]  # keep the FP32 outputs of the caller
    out = {"pairs": n, "reference": "FP64 device solve of the same schedule (the only FP64 path)"}
    for name, st in (("fp32", rf.STORE_FP32), ("fp16", rf.STORE_FP16), ("bf16", rf.STORE_BF16)):
        prm = rf.benchmark_params(W)
        prm.storage = st
        fl = ctx.scene_flow_batch(host, prm, stats=False)
        e64, e32 = epes(fl, f64), epes(fl, f32)
        # device-resident throughput and per-kernel-class GB/s of the stored type
        for _ in range(2):
            ctx.scene_flow_batch_device(dev, prm)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            ctx.scene_flow_batch_device(dev, prm)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        ctx.profile(1)
        ctx.scene_flow_batch_device(dev, prm)
        torch.cuda.synchronize()
        kst = ctx.profile_read()
        ctx.profile(0)
        gbs = {k: kst[k][2] / (kst[k][1] / 1e3) / 1e9 for k in ("sor", "linearize") if k in kst and kst[k][1] > 0}
        out[name] = {"pairs_per_s": 1e3 * len(dev) / ms,
                     "epe_vs_fp64_mm": {"mean": 1e3 * float(np.mean([e[0] for e in e64])),
                                        "max": 1e3 * float(np.max([e[1] for e in e64]))},
                     "epe_vs_fp32_mm": {"mean": 1e3 * float(np.mean([e[0] for e in e32])),
                                        "max": 1e3 * float(np.max([e[1] for e in e32]))},
                     "algorithmic_gbs": gbs}
    return out


def cpu_baselines(host, dev, torch):
    """The CPU restatement of the reference (oracle, all host threads) at 640x480 and at 320x240
    (the reference's CPU-runnable configuration), median of 5 solves each; beside it the
    reference's own CUDA solver (sceneFlowSingleScaleJacobiCUDA.cu, compiled for sm_100a) driven
    level by level with pyramids, features and warps on the host, as the reference runs."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    import rgbdflow as rf
    ob.build_oracle()
    threads = ob.oracle().sfo_set_threads(0)

    def timed(p, n, ref_cuda=False):
        prm = rf.benchmark_params(p["W"])
        cam = cam_of(rf, p)
        ts, out = [], None
        for _ in range(n):
            t = time.perf_counter()
            if ref_cuda:
                with ob.reference_cuda_levels():
                    out, _ = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
            else:
                out, _ = ob.two_frames(cam, p["bgr1"], p["depth1"], p["bgr2"], p["depth2"], prm)
            ts.append(time.perf_counter() - t)
        return float(np.median(ts)), out

    p640 = host[0]
    p320 = syn.make_config_pair("320x240", seed=1)
    t640, o640 = timed(p640, 5)
    t320, _ = timed(p320, 5)
    gpu0 = dev[0]["out"].cpu().numpy()
    mask = p640["depth1"] > 0
    mean, mx = syn.epe3d(gpu0, o640, p640["z1_true"], p640["cam"], mask)
    cpu = {"value": 1.0 / t640, "unit": "pairs/s", "cores": threads, "kind": "port",
           "sample": "5 solves of one 640x480 pair, median (the oracle, OpenMP over rows)",
           "config_320x240": {"pairs_per_s": 1.0 / t320, "ms": 1e3 * t320, "sample": "5 solves, median"},
           "epe_vs_gpu_mm": {"mean": mean * 1e3, "max": mx * 1e3}}
    if ob.ref_cuda_available():
        try:
            r640, q640 = timed(p640, 3, ref_cuda=True)
            r320, _ = timed(p320, 3, ref_cuda=True)
            m2, x2 = syn.epe3d(gpu0, q640, p640["z1_true"], p640["cam"], mask)
            cpu["reference_cuda"] = {
                "what": "the reference's own CUDA solver (sceneFlowSingleScaleJacobiCUDA.cu, sm_100a build) per "
                        "level, pyramids / features / warps on the host cores, as the reference runs; 3 solves, median",
                "pairs_per_s_640x480": 1.0 / r640, "pairs_per_s_320x240": 1.0 / r320,
                "epe_vs_gpu_mm": {"mean": m2 * 1e3, "max": x2 * 1e3}}
        except Exception as e:  # the reference solver is a baseline only; report why it is missing
            cpu["reference_cuda"] = {"unavailable": str(e)[:200]}
    torch.cuda.synchronize()
    return cpu


def bench_config(rf, B, world):
    """The workload both arms report: B independent 640x480 pairs per step per GPU, with the batch's
    solve memory (host-computed from the plan) as the working set against the 126 MB L2."""
    ws = rf.batch_device_bytes([(W, H)] * B, rf.benchmark_params(W))
    return {"workload": "batched solve of %d independent 640x480 pairs per step per GPU (5 levels x 10 outer "
                        "x 30 SOR, reference convergence breaks)" % B,
            "global_batch": B * world, "parallelism": "replicas x%d" % world,
            "l2": "inputs larger than L2 (working set %.2f GB per GPU)" % (ws / 1e9)}


def run_reference(args, rank, world):
    """The reference arm: the reference has no CPU implementation of its 3-D solver, so its
    restatement (oracle/, the same arithmetic and schedule) runs on the host cores."""
    if rank != 0:
        return
    import rgbdflow as rf
    # the pairs of the device arm's batch (rank 0's seeds), as many as the timed steps visit
    pairs = make_pairs(max(1, min(args.batch, args.steps)), 0)
    if args.warmup:
        oracle_pairs_per_s(pairs, min(args.warmup, 1))
    v, threads, _, ts = oracle_pairs_per_s(pairs, args.steps)
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(ts)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 (mixed, as the reference)",
            "data": "synthetic (seeded RGB-D patch scenes, 640x480)",
            "config": bench_config(rf, args.batch, world),
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": threads, "kind": "port",
                             "sample": "%d pairs of the device arm's 640x480 batch, one per step (the CPU "
                                       "restatement of the reference on the host cores)" % args.steps},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the served load sweep")
    ap.add_argument("--no-flow2d", action="store_true", help="skip the 2-D optical flow timing")
    ap.add_argument("--serve-frames", type=int, default=150)
    ap.add_argument("--serve-unique", type=int, default=8)
    ap.add_argument("--ncu-case", type=int, default=0, metavar="NP",
                    help="profiling case: one batched solve of NP 640x480 pairs with graphs off "
                         "(every launch visible to a profiler), then exit; prints no bench line")
    ap.add_argument("--ncu-storage", default="fp32", choices=["fp32", "fp16", "bf16"],
                    help="storage type of the feature / depth pyramids in the profiling case")
    ap.add_argument("--ncu-reg", default="isotropic", choices=["isotropic", "letouzey", "hpb"],
                    help="regularisation of the profiling case")
    ap.add_argument("--ncu-flow2d", default="", choices=["", "320x240", "640x480"],
                    help="profiling case: one 2-D optical flow (the demo's flow type 1) of the synthetic "
                         "pair of this size, then exit; prints no bench line")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    if args.ncu_case:
        os.environ["RGBDFLOW_NO_GRAPHS"] = "1"  # read when the context is created
    import torch
    import torch.distributed as dist
    import rgbdflow as rf

    torch.cuda.set_device(local)
    if args.ncu_case:
        run_ncu_case(args.ncu_case, rf, torch, args.ncu_storage, args.ncu_reg)
        return
    if args.ncu_flow2d:
        p = syn.make_config_pair(args.ncu_flow2d, seed=1)
        c = rf.Context(local)
        c.optical_flow_2d(p["bgr1"], p["bgr2"])
        c.close()
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    import replicas

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, device="cuda")

    B = args.batch
    host = make_pairs(B, replicas.pair_seed(rank, 0))
    prm = rf.benchmark_params(W)
    ctx = rf.Context(local)
    dev = [device_pair(rf, torch, p) for p in host]
    stream = torch.cuda.Stream()  # the stream every solve below is enqueued on and timed on
    torch.cuda.set_stream(stream)

    # ---- value: device-resident batched solves, LANES batches in flight.  Steps rotate over LANES
    # contexts on as many streams; before a context takes its next step the host waits for its
    # previous one, so the batches run a fraction of a solve apart and one batch's SM-saturating
    # 640x480-level SOR overlaps the others' latency-bound coarse levels (1, 2, 3 and 4 in
    # flight: 645, 743, 752 and 761 pairs/s).  Timed on the device: from an event every stream
    # waits on to the latest of the streams' last events.
    lanes = [(ctx, stream, dev)]
    for _ in range(LANES - 1):
        lanes.append((rf.Context(local), torch.cuda.Stream(), [dict(d, out=torch.empty_like(d["out"])) for d in dev]))

    def timed_steps(n_steps, multi):
        nl = LANES if multi else 1
        done = [None] * nl
        starts, ends = [], []
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _, st, _ in lanes[1:]:
            st.wait_event(e0)
        for s in range(n_steps):
            c, st, dv = lanes[s % nl]
            if done[s % nl] is not None:
                done[s % nl].synchronize()
            a = torch.cuda.Event(enable_timing=True)
            a.record(st)
            c.scene_flow_batch_device(dv, prm, stream=st)
            b = torch.cuda.Event(enable_timing=True)
            b.record(st)
            done[s % nl] = b
            starts.append(a)
            ends.append(b)
        for d in done:
            if d is not None:
                stream.wait_event(d)
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), [a.elapsed_time(b) for a, b in zip(starts, ends)]

    timed_steps(max(args.warmup, LANES), True)
    launches_per_step = ctx.last_launch_count()
    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    ms_raw, step_ms = timed_steps(args.steps, True)
    barrier()
    clk = clocks.stop()
    ms = max_over_ranks(ms_raw)
    value = replicas.aggregate_rate(B * args.steps, world, ms / 1e3)
    # the same steps one batch at a time (a step's latency without overlap), for comparison
    ms1_raw, step1_ms = timed_steps(args.steps, False)
    value_one = replicas.aggregate_rate(B * args.steps, world, max_over_ranks(ms1_raw) / 1e3)
    for c, _, _ in lanes[1:]:
        c.close()

    # ---- batched result check: pair 0 of the batch equals the same pair solved alone
    solo = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    d0 = dict(dev[0])
    d0["out"] = solo
    ctx.scene_flow_batch_device([d0], prm)
    torch.cuda.synchronize()
    same = bool(torch.equal(solo, dev[0]["out"]))

    # ---- plain: one pair per call (the drop-in form), per-call latency
    lat = []
    for s in range(0 if args.no_plain else max(args.warmup, 2) + 20):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ctx.scene_flow_batch_device([dev[s % B]], prm)
        b.record(stream)
        torch.cuda.synchronize()
        if s >= max(args.warmup, 2):
            lat.append(a.elapsed_time(b))
    plain = None
    if lat:
        plain = {"pairs_per_s": 1e3 / float(np.mean(lat)), "p50_ms": float(np.percentile(lat, 50)),
                 "p99_ms": float(np.percentile(lat, 99)), "calls": len(lat)}

    # ---- e2e: host buffers through the synchronous C ABI call
    # inputs and outputs in page-locked host memory: the library DMAs them directly
    def pinned(a):
        t = torch.from_numpy(a).pin_memory()
        return t.numpy()
    hp = [dict(W=W, H=H, cam=cam_of(rf, p), bgr1=pinned(p["bgr1"]), depth1=pinned(p["depth1"]),
               bgr2=pinned(p["bgr2"]), depth2=pinned(p["depth2"])) for p in host]
    pouts = [torch.empty((H, W, 3), dtype=torch.float32).pin_memory().numpy() for _ in host]
    e2e = None
    if not args.no_e2e:
        # LANES contexts rotate, as for the device-resident value: step s uploads its inputs,
        # solves and downloads its flows on one context (rgbdflow_scene_flow_batch_submit returns
        # once enqueued) while the other contexts' steps run; a context is synchronised (its flows
        # read) before it takes its next step
        ctxs = [ctx] + [rf.Context(local) for _ in range(LANES - 1)]
        outs2 = [pouts] + [[torch.empty((H, W, 3), dtype=torch.float32).pin_memory().numpy() for _ in host]
                           for _ in range(LANES - 1)]

        def e2e_step(s):
            c = ctxs[s % LANES]
            if s >= LANES:
                c.synchronize()
            c.scene_flow_batch_submit(hp, prm, outs2[s % LANES])

        for s in range(max(args.warmup, LANES)):
            e2e_step(s)
        for c in ctxs:
            c.synchronize()
        barrier()
        t = time.perf_counter()
        for s in range(args.steps):
            e2e_step(s)
        for c in ctxs:
            c.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t)
        for c in ctxs[1:]:
            c.close()
        e2e = {"value": B * args.steps * world / e2e_s, "unit": "pairs/s",
               "h2d_bytes_per_step": B * W * H * (3 + 3 + 4 + 4), "d2h_bytes_per_step": B * W * H * 12,
               "how": "rgbdflow_scene_flow_batch_submit on %d contexts in rotation: each step uploads its "
                      "inputs from page-locked host memory, solves, and downloads its flows; one step's transfers "
                      "overlap the other contexts' solves" % LANES}

    # ---- roofline of the dominant kernel from a profiled pass of the same workload: the SOR of
    # the 640x480 level (the strip kernel), algorithmic bytes / live CUDA-event time
    ctx.profile(1)
    for _ in range(2):
        ctx.scene_flow_batch_device(dev, prm)
    torch.cuda.synchronize()
    kst = ctx.profile_read()
    ctx.profile(0)
    peak, peak_kind = peaks()
    n0, ms0, b0 = kst.get("sor_level0", (0, 0.0, 0.0))
    n_sor, sor_ms, sor_bytes = kst.get("sor", (0, 0.0, 0.0))
    achieved = b0 / (ms0 / 1e3) / 1e9 if ms0 > 0 else 0.0
    tr = ncu_traffic()
    tot_ms = sum(v[1] for k, v in kst.items() if not k.startswith("sor_level"))
    roofline = {"kernel": "k_sor_strip: red-black SOR of the 640x480 level over 64-column strips, rows streamed "
                          "through a shared-memory ring, 5 sweeps per launch",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "traffic": (tr["dram_bytes_per_launch_per_pair"] * B if tr else None),
                "algorithmic_bytes_per_launch": b0 / max(n0, 1),
                "avg_launch_us": 1e3 * ms0 / max(n0, 1), "launches": n0,
                "share_of_device_time": ms0 / tot_ms if tot_ms else None,
                "all_sor_levels": {"achieved_gbs": sor_bytes / (sor_ms / 1e3) / 1e9 if sor_ms > 0 else 0.0,
                                   "frac": (sor_bytes / (sor_ms / 1e3) / 1e9) / peak if sor_ms > 0 else 0.0,
                                   "share_of_device_time": sor_ms / tot_ms if tot_ms else None},
                "kernel_ms": {k: round(v[1], 3) for k, v in kst.items()}}
    if tr:
        roofline["traffic_note"] = tr.get("note", "")

    # ---- served: camera streams at 30 fps (Poisson arrivals) through the continuous-batching
    # server.  Headline: cold pairs (the full coarse-to-fine solve, the same flow as the plain
    # call); beside it, warm starts from each stream's previous flow.
    served = served_warm = None
    if not args.no_serve:
        import serving
        streams = serving.make_streams(n_unique=args.serve_unique, seed0=500 + 100 * rank)
        served = run_served(ctx, rf, serving, streams, prm, args, warm=False)
        served_warm = run_served(ctx, rf, serving, streams, prm, args, warm=True)
        if not args.no_sweep:
            pts = [(n, 30) for n in (8, 10, 12, 14, 16, 18, 20, 24, 32, 40, 48)]
            served["capacity"] = run_served_sweep(ctx, rf, serving, streams, prm, False, pts)
            served_warm["capacity"] = run_served_sweep(ctx, rf, serving, streams, prm, True, pts)

    # ---- batching: the uneven mix of 64 pairs (24 x 160x120, 24 x 320x240, 16 x 640x480) in one
    # persistent launch per pyramid level
    mixed = None if args.no_mixed else run_mixed(ctx, rf, torch, stream, prm, args, rank)

    # ---- precision: pyramids stored in FP16 / BF16 (flow and Jacobi accumulation in FP32),
    # against the FP32 and the FP64 device solves of the same pairs
    precision = None if args.no_precision else run_precision(ctx, rf, torch, stream, dev, host, args)

    # ---- the demo's 2-D optical flow (flow type 1): ms per pair through the host-buffer call,
    # beside the CPU restatement at 320x240 (FP64 lexicographic SOR, one thread)
    flow2d = None
    if rank == 0 and not args.no_flow2d:
        flow2d = {}
        for name in ("320x240", "640x480"):
            p = syn.make_config_pair(name, seed=1)
            ctx.optical_flow_2d(p["bgr1"], p["bgr2"])
            ts = []
            for _ in range(2):
                t = time.perf_counter()
                f2 = ctx.optical_flow_2d(p["bgr1"], p["bgr2"])
                ts.append(time.perf_counter() - t)
            flow2d["gpu_ms_" + name] = 1e3 * min(ts)
            if name == "320x240" and world == 1 and not args.no_cpu_baseline:
                sys.path.insert(0, os.path.join(ROOT, "tests"))
                import oracle_binding as ob
                t = time.perf_counter()
                u, v = ob.optical_flow_2d(p["bgr1"], p["bgr2"])
                flow2d["cpu_ms_320x240"] = 1e3 * (time.perf_counter() - t)
                flow2d["gpu_equals_cpu_320x240"] = bool(np.array_equal(f2, np.stack([u, v], -1).astype(np.float32)))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baselines(host, dev, torch)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded RGB-D patch scenes, 640x480)",
                "config": bench_config(rf, B, world),
                "batches_in_flight": LANES,
                "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
                "one_batch_in_flight": {"value": value_one, "p50_ms": float(np.percentile(step1_ms, 50)),
                                        "p99_ms": float(np.percentile(step1_ms, 99))},
                "plain": plain, "batch_equals_solo": same, "served": served, "served_warm": served_warm,
                "mixed_batch": mixed, "precision": precision, "flow2d": flow2d,
                "gpu_launches": launches_per_step * args.steps,
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "autotune": rf.autotune_describe(local)}
        print(json.dumps(compact(line)), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
