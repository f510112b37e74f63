#!/usr/bin/env python
"""Benchmark of the XnYZip compress + decompress path on B200.

Workload (N=1): the terrain-LiDAR cloud of the plain method - 64M float32 points (x,y
uniform over [0,10000]^2 m, 8 sinusoid octaves + N(0,0.1^2) noise, 5% multi-return
copies), Hilbert curve, -rle container, both quantizers (to, cube) x L2 bounds
{0.001, 0.01, 0.1}.  One step = compress + decompress of the cloud for all six variants.

  value : compress+decompress GB/s (12 bytes per input point) with the points resident in
          HBM, the pre-zstd container produced and consumed in HBM (xnyz_compress_device /
          xnyz_decompress_device), device time from CUDA events on the library's stream; the
          variants, which are independent, run on --pipes contexts (streams) from host threads
          so that one variant's kernels fill another's gaps.
  e2e   : the same through the host-buffer C ABI, batched (xnyz_batch_compress /
          xnyz_batch_decompress: worker threads with one context each): pinned host points
          in, the reference's zstd level-3 frames out (libzstd 1.5.7 on the host), frames in,
          pinned host points out; wall clock with device sync on both sides.  The headline
          cuts the cloud into --chunk-point pieces, one frame each, exactly the workload the
          reference arm runs; `monolithic` is one frame per variant for the whole cloud.
  bits/point per variant from the zstd frame.
  roofline: the dominant stage of one extra (untimed) step profiled with per-stage CUDA
          events and side-stream work serialised (xnyz_profile mode 2).
  learned : the extended container on the same cloud (block parameters of the repos /
          SFC-delta stream: reference coding, one global pair, learned, exhaustive): pre-zstd
          bits/point, penalty against exhaustive search, device GB/s against plain.
  batched : the uneven batch (2048 clouds, ~1e9 points, log-uniform sizes), per-cloud plain
          launches on one context against xnyz_batch_roundtrip_device (autotuned worker
          streams per size class), with the reference container and with learned parameters.

spheres : the clustered-surface cloud (175M points on 200,000 spheres, TO, L2 0.5, Morton,
          -normal and -rle), device GB/s and parity in its own sub-line (--no-spheres skips it);
          --workload spheres makes it the main workload instead.

--gpus N: one process per GPU (torchrun); the path does not shard, every rank runs its
own replica on its own cloud (seed 1 + rank): weak scaling, max time over ranks.

--impl reference: the reference's own CPU implementation (oracle/_ref, built from its
sources; the oracle restatement if absent) over all host threads, each thread compressing
and decompressing its own chunk of the same workload (the reference's per-chunk mode).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# workloads: (generator, default points, [(quantizer, l2, hilbert, rle)])
WORKLOADS = {
    # terrain-LiDAR plain method: both quantizers x L2 {0.001, 0.01, 0.1}, Hilbert, -rle
    "terrain": ("terrain", 64_000_000, [(1, 0.001, 1, 1), (1, 0.01, 1, 1), (1, 0.1, 1, 1),
                                        (0, 0.001, 1, 1), (0, 0.01, 1, 1), (0, 0.1, 1, 1)]),
    # clustered surfaces: 200,000 spheres, TO, L2 0.5, Morton, -normal and -rle
    "spheres": ("spheres", 175_000_000, [(1, 0.5, 0, 0), (1, 0.5, 0, 1)]),
}


def vname(v):
    q, l2, hil, rle = v
    return f"{QNAME[q]}_{l2}" + ("" if (hil, rle) == (1, 1) else f"_{'h' if hil else 'z'}_{'rle' if rle else 'normal'}")
QNAME = {0: "cube", 1: "to"}
# DRAM bytes (read + write) per key of one keys-only sort pass, from an ncu capture of one
# sort_pass_kernel<0> launch over 24M terrain keys (199.4 MB read + 154.5 MB written): below
# the 16 algorithmic bytes because part of the input is still in L2 from the previous pass.
# Scaled by the keys of a launch; the L2 share shrinks as the cloud grows, so at 64M keys
# this is a lower bound on the traffic.
SORT_PASS_DRAM_BYTES_PER_KEY = (199.396608e6 + 154.480640e6) / 24e6
METRIC = "compress+decompress GB/s (12 B/point input) at fixed L2 bound"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def _synthetic():
    """The seeded generators, loaded from their file: importing the package would load the
    CUDA library, which the reference arm must not map."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("xnyz_synthetic", os.path.join(ROOT, "xnyzip_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cloud_seed(workload: str, rank: int) -> int:
    """Seed of rank `rank`'s cloud (the terrain cloud of rank 0 is seed 1, the spheres seed 2)."""
    return 1 + rank + (1 if WORKLOADS[workload][0] == "spheres" else 0)


def make_cloud(workload: str, n: int, seed: int):
    S = _synthetic()
    if WORKLOADS[workload][0] == "spheres":
        return S.spheres(n, 200_000, seed)
    return S.terrain(n, seed)


def workload_config(workload: str, n: int, variants, world: int = 1) -> dict:
    """The bench line's config, the same for both arms."""
    return {
        "workload": (f"terrain {n} points, Hilbert, -rle, quantizers to/cube x L2 {{0.001,0.01,0.1}}"
                     if workload == "terrain" else
                     f"spheres {n} points on 200,000 spheres, TO, L2 0.5, Morton, -normal and -rle")
                    + f"; one step = compress+decompress of all {len(variants)} variants",
        "points": n,
        "variants": [vname(v) for v in variants],
        "direct_threshold": 1024,
        "l2_flush": f"inputs ({12 * n / 1e6:.0f} MB per cloud) exceed the 126 MB L2",
        "parallelism": f"replicas x{world}",
    }


def load_digests() -> dict:
    """Reference digests of the full-size clouds (tests/golden/make_ref_digests.py)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "ref_digests.json")) as f:
            return json.load(f)
    except FileNotFoundError:
        return {}


class RankSync:
    """Barrier and max-over-ranks of a timing: one value per rank, the job's time is the
    slowest rank's.  NCCL with a device tensor on GPUs, gloo with a host tensor elsewhere."""

    def __init__(self, world: int, device=None):
        self.world = world
        self.device = device

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())


# ------------------------------------------------------------------------------ GPU arm ---
def run_gpu(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import xnyzip_b200 as X

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # A dedicated stream shared with the library: the timing events below are recorded on
    # the stream the kernels are launched on.
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = X.Context(local, stream=stream.cuda_stream)

    n = args.points or WORKLOADS[args.workload][1]
    t0 = time.time()
    seed = cloud_seed(args.workload, rank)
    host = make_cloud(args.workload, n, seed)
    log(f"[rank {rank}] generated {n} points in {time.time() - t0:.1f}s")
    pinned = torch.from_numpy(host).pin_memory()
    d_pts = pinned.to(dev, non_blocking=False)
    torch.cuda.synchronize(dev)
    variants = WORKLOADS[args.workload][2][: args.variants]

    sync = RankSync(world, dev)
    barrier = sync.barrier
    max_over_ranks = sync.max

    # ---- device-resident step ----
    def run_variants(c, vs):
        lens = []
        for q, l2, hil, rle in vs:
            p, ln = c.compress_device(d_pts.data_ptr(), n, q, l2, hil, rle)
            lens.append(ln)
            _, nout = c.decompress_device(p, ln, q, l2, rle)
            if nout != n:
                raise RuntimeError(f"decoded {nout} points, expected {n}")
        return lens

    def serial_step():  # every variant on the one context (the profiled step)
        return run_variants(ctx, variants)

    # The timed step runs the variants, which are independent, on `pipes` contexts with their
    # own streams from host threads, so that one variant's kernels fill the gaps of another's
    # (its host-side codebook work, latency-bound decoders).  The other streams wait for an
    # event on the main stream before their first call and the main stream waits for theirs
    # at the end: the CUDA events on the main stream bracket all of the step's work.
    pipes = max(1, min(args.pipes, len(variants)))
    pipe_streams = [stream] + [torch.cuda.Stream(dev) for _ in range(pipes - 1)]
    pipe_ctx = [ctx] + [X.Context(local, stream=s.cuda_stream) for s in pipe_streams[1:]]

    def device_step():
        if pipes == 1:
            return serial_step()
        start = torch.cuda.Event()
        start.record(stream)
        for s in pipe_streams[1:]:
            s.wait_event(start)
        out, errs = [None] * pipes, []

        def worker(k):
            try:
                out[k] = run_variants(pipe_ctx[k], variants[k::pipes])
            except Exception as e:  # re-raised on the main thread
                errs.append(e)

        ths = [threading.Thread(target=worker, args=(k,)) for k in range(pipes)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        if errs:
            raise errs[0]
        for s in pipe_streams[1:]:
            done = torch.cuda.Event()
            done.record(s)
            stream.wait_event(done)
        lens = [0] * len(variants)
        for k in range(pipes):
            lens[k::pipes] = out[k]
        return lens

    for _ in range(args.warmup):
        clens = device_step()
    barrier()
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        clens = device_step()
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    dev_ms = ev0.elapsed_time(ev1)
    dev_ms = max_over_ranks(dev_ms)
    barrier()
    # one more step with per-stage CUDA events, the side streams' work issued on the context's
    # stream (xnyz_profile mode 2), so that each stage's time is its own: the roofline
    for c in pipe_ctx[1:]:  # their workspaces are not needed past the timed step
        c.close()
    ctx.profile(2)
    serial_step()
    prof_all = ctx.profile_read()
    ctx.profile(False)
    prof = {k: v for k, v in prof_all.items() if not k.startswith("host:")}
    host_phases = {k[5:]: round(v["ms"], 3) for k, v in prof_all.items() if k.startswith("host:")}
    torch.cuda.synchronize(dev)
    barrier()

    # ---- end-to-end through the host-buffer C ABI: batches of independent calls ----
    # Pinned host points in, zstd frames out, frames in, pinned host points out; each step
    # (1) the cloud in `chunk`-point pieces for all variants, the reference arm's per-chunk
    # workload (headline), and (2) the whole cloud once per variant (one frame each).
    batch = X.Batch(local, args.workers)
    host_np = pinned.numpy()
    outs = [torch.empty((n, 3), dtype=torch.float32).pin_memory().numpy() for _ in variants]
    bounds = [(a, min(n, a + args.chunk)) for a in range(0, n, args.chunk)]
    c_clouds = [host_np[a:b] for _ in variants for (a, b) in bounds]
    c_params = [(q, l2, hil, rle) for (q, l2, hil, rle) in variants for _ in bounds]
    c_dparams = [(q, l2, rle) for (q, l2, hil, rle) in variants for _ in bounds]
    c_outs = [outs[vi][a:b] for vi in range(len(variants)) for (a, b) in bounds]
    m_clouds = [host_np for _ in variants]
    m_params = [(q, l2, hil, rle) for (q, l2, hil, rle) in variants]
    m_dparams = [(q, l2, rle) for (q, l2, hil, rle) in variants]
    frame_bytes = {}
    chunk_bytes = {}

    def e2e_chunked_step():
        if args.e2e_mode == "roundtrip":  # each chunk's compress + decompress on one worker
            frames = batch.roundtrip(c_clouds, c_params, c_outs)
        else:  # every compress, then every decompress
            frames = batch.compress(c_clouds, c_params, as_bytes=False)
            ns = batch.decompress(frames, c_dparams, c_outs)
            if ns != [b - a for _ in variants for (a, b) in bounds]:
                raise RuntimeError("e2e (chunked) decode size mismatch")
        for vi, v in enumerate(variants):
            chunk_bytes[v] = sum(len(f) for f in frames[vi * len(bounds):(vi + 1) * len(bounds)])

    mono_frames = {}

    def e2e_monolithic_step():
        if args.e2e_mode == "roundtrip":
            frames = batch.roundtrip(m_clouds, m_params, outs)
        else:
            frames = batch.compress(m_clouds, m_params, as_bytes=False)
            ns = batch.decompress(frames, m_dparams, outs)
            if ns != [n] * len(variants):
                raise RuntimeError("e2e decode size mismatch")
        for v, f in zip(variants, frames):
            frame_bytes[v] = len(f)
            mono_frames[v] = f  # the last step's frames are checked against the reference below

    def timed(fn, steps):
        fn()  # warm-up: worker arenas and pinned staging reach their sizes
        barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for _ in range(steps):
            fn()
        torch.cuda.synchronize(dev)
        return max_over_ranks(time.perf_counter() - w0)

    e2e_steps = min(args.steps, args.e2e_steps)  # 0: skip (device-only profiling runs)
    if e2e_steps:
        e2e_s = timed(e2e_chunked_step, e2e_steps)
        mono_s = timed(e2e_monolithic_step, e2e_steps)
    batch.close()

    # ---- parity of the timed paths with the reference, and the L2 bound of every point ----
    parity = None
    if args.parity and rank == 0:
        parity = parity_measure(ctx, dev, d_pts, host, n, variants, args.workload, seed,
                                mono_frames if e2e_steps else None, outs if e2e_steps else None)
    del outs, mono_frames

    # ---- learned block parameters (extended container) on the same cloud ----
    learned = None
    if args.learned and rank == 0:
        learned = learned_measure(ctx, stream, d_pts, n, variants, args.steps)
        learned["mlp_kernels"] = mlp_measure(dev, stream)

    # ---- the uneven batch (2048 clouds): per-cloud plain launches vs the batched path ----
    batched = None
    if args.batch_clouds and rank == 0 and world == 1:
        batched = batched_measure(ctx, stream, dev, args.batch_clouds, args.workers)

    # ---- the clustered-surface cloud (175M points on 200,000 spheres), its own sub-line ----
    spheres = None
    if args.spheres and args.workload == "terrain" and rank == 0 and world == 1:
        try:
            spheres = spheres_measure(ctx, stream, dev, min(args.steps, 3), args.warmup, args.parity)
        except Exception as e:  # reported in the line, the rest of it stands
            spheres = {"error": f"{type(e).__name__}: {e}"}

    # ---- zstd frames decoded on the GPU ----
    zstd_frames = None
    if args.zstd_frames and rank == 0 and world == 1:
        try:
            zstd_frames = zstd_measure(ctx, stream, dev, count=args.zstd_frames)
        except Exception as e:  # reported in the line, the rest of it stands
            zstd_frames = {"error": f"{type(e).__name__}: {e}"}

    # ---- CPU baseline: the reference on a bounded sample (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(host, variants, args.cpu_points, threads=1)

    if rank == 0:
        bytes_step = 12.0 * n * len(variants) * world
        value = bytes_step * args.steps / (dev_ms / 1e3) / 1e9
        e2e = bytes_step * e2e_steps / e2e_s / 1e9 if e2e_steps else None
        mono = bytes_step * e2e_steps / mono_s / 1e9 if e2e_steps else None
        peak, peak_kind = load_peaks()
        # dominant kernel: largest total device time among the profiled stages
        dom_name, dom = max(prof.items(), key=lambda kv: kv[1]["ms"])
        per_launch_ms = dom["ms"] / max(1, dom["launches"])
        per_launch_bytes = dom["bytes"] / max(1, dom["launches"])
        achieved = per_launch_bytes / (per_launch_ms / 1e3) / 1e9
        stage_bytes = sum(v["bytes"] for v in prof.values())
        stage_ms = sum(v["ms"] for v in prof.values())
        launches = sum(v["launches"] for v in prof.values()) * args.steps  # prof covers one step
        bpp = {vname(v): round(8.0 * frame_bytes[v] / n, 4) for v in variants if v in frame_bytes}
        line = {
            "metric": METRIC,
            "value": round(value, 3),
            "unit": "GB/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(dev_ms / args.steps, 3),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 in, int32/u64 lattice and key arithmetic",
            "data": (f"synthetic {'terrain-LiDAR' if args.workload == 'terrain' else 'clustered-surface'} "
                     f"stand-in (seeded, {n} points), generated on the host"),
            "config": workload_config(args.workload, n, variants, world),
            "paths": {
                "value": f"device-resident points and pre-zstd container; the independent variants spread "
                         f"over {pipes} contexts / streams, CUDA events on the main stream bracketing all",
                "e2e": "pinned host points -> zstd frames (libzstd 1.5.7 level 3) -> pinned host points, "
                       + ("xnyz_batch_roundtrip (each chunk's pair on one worker)" if args.e2e_mode == "roundtrip"
                          else "xnyz_batch_compress then xnyz_batch_decompress"),
            },
            "bits_per_point": bpp,
            "e2e": ({"value": round(e2e, 4), "unit": "GB/s", "h2d_bytes_per_step": int(12 * n * len(variants)),
                     "d2h_bytes_per_step": int(12 * n * len(variants)), "steps": e2e_steps,
                     "s_per_step": round(e2e_s / e2e_steps, 4),
                     "workload": f"{len(bounds)} chunks of {args.chunk} points x {len(variants)} variants "
                                 f"(the reference arm's per-chunk mode), one zstd frame per chunk, "
                                 f"xnyz_batch_* with {batch.workers} worker threads",
                     "bits_per_point": {vname(v): round(8.0 * chunk_bytes[v] / n, 4) for v in variants},
                     "monolithic": {"value": round(mono, 4), "unit": "GB/s", "s_per_step": round(mono_s / e2e_steps, 4),
                                    "workload": "the whole cloud, one zstd frame per variant, "
                                                f"{len(variants)} variants in one batch"}}
                    if e2e_steps else None),
            "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1), "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": (round(SORT_PASS_DRAM_BYTES_PER_KEY * per_launch_bytes / 16.0)
                                     if dom_name == "sort_pass" and per_launch_bytes and args.workload == "terrain"
                                     else None),
                         "traffic_source": "ncu DRAM bytes per key of a keys-only pass over 24M keys, "
                                           "scaled to this launch's keys",
                         "bytes_per_launch": per_launch_bytes, "ms_per_launch": round(per_launch_ms, 4),
                         "pipeline_achieved": round(stage_bytes / (stage_ms / 1e3) / 1e9, 1),
                         "pipeline_frac": round(stage_bytes / (stage_ms / 1e3) / 1e9 / peak, 4)},
            "stages": {k: {"ms_per_step": round(v["ms"], 4), "launches": v["launches"],
                           "GB_s": round(v["bytes"] / (v["ms"] / 1e3) / 1e9, 1) if v["ms"] else None}
                       for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])},
            "stages_note": "one extra step (not timed) with per-stage CUDA events, side-stream work serialised",
            "host_phases_ms_per_step": host_phases,
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if parity is not None:
            line["parity"] = parity.pop("per_variant")
            line["parity_detail"] = parity
        if learned is not None:
            line["learned"] = learned
        if batched is not None:
            line["batched"] = batched
        if spheres is not None:
            line["spheres"] = spheres
        if zstd_frames is not None:
            line["zstd_frames"] = zstd_frames
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# -------------------------------------------------------------------- spheres (config 3) ---
def spheres_measure(ctx, stream, dev, steps, warmup, check_parity, n=175_000_000):
    """The clustered-surface plain method (175M points on 200,000 spheres, TO, L2 0.5, Morton,
    -normal and -rle): device-resident compress+decompress GB/s of both variants, each on its
    own context and stream (CUDA events on `stream` bracket both), max-over-nothing (one
    rank), and the same parity checks as the main workload against the reference's digests
    of this cloud."""
    import threading as th
    import torch
    import xnyzip_b200 as X
    t0 = time.time()
    host = make_cloud("spheres", n, cloud_seed("spheres", 0))
    gen_s = time.time() - t0
    d_pts = torch.from_numpy(host).to(dev)
    torch.cuda.synchronize(dev)
    variants = WORKLOADS["spheres"][2]
    side = torch.cuda.Stream(dev)
    ctx2 = X.Context(dev.index, stream=side.cuda_stream)
    ctxs = [ctx, ctx2]
    streams = [stream, side]

    def one(c, v):
        q, l2, hil, rle = v
        p, ln = c.compress_device(d_pts.data_ptr(), n, q, l2, hil, rle)
        _, nout = c.decompress_device(p, ln, q, l2, rle)
        if nout != n:
            raise RuntimeError(f"decoded {nout} points, expected {n}")

    def step():
        start = torch.cuda.Event()
        start.record(stream)
        side.wait_event(start)
        errs = []

        def work(i):
            try:
                one(ctxs[i], variants[i])
            except Exception as e:  # re-raised below
                errs.append(e)

        ts = [th.Thread(target=work, args=(i,)) for i in range(2)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if errs:
            raise errs[0]
        done = torch.cuda.Event()
        done.record(side)
        stream.wait_event(done)

    for _ in range(max(1, warmup)):
        step()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    ctx2.close()
    out = {"workload": f"spheres {n} points on 200,000 spheres, TO, L2 0.5, Morton; one step = compress+decompress "
                       "of the -normal and the -rle variant, one context / stream each",
           "points": n, "variants": [vname(v) for v in variants], "steps": steps, "warmup": max(1, warmup),
           "ms_per_step": round(ms, 3), "GB_s": round(12.0 * n * len(variants) / (ms / 1e3) / 1e9, 3),
           "generate_s": round(gen_s, 1)}
    if check_parity:
        par = parity_measure(ctx, dev, d_pts, host, n, variants, "spheres", cloud_seed("spheres", 0), None, None)
        out["parity"] = par.pop("per_variant")
        out["parity_detail"] = par
    del d_pts, host
    torch.cuda.empty_cache()
    return out


# ----------------------------------------------------------------------------- parity ---
def parity_measure(ctx, dev, d_pts, host, n, variants, workload, seed, mono_frames, mono_outs):
    """The timed paths' outputs against the reference's, at full size, after the timed region.

    Per variant: the device container (xnyz_compress_device), the zstd frame of the
    host-output call (xnyz_compress from the resident points), the device decode
    (xnyz_decompress_device), and the last e2e step's whole-cloud frame and host points, each
    by SHA-256 against tests/golden/ref_digests.json (the reference run on the same seeded
    cloud); and the L2 report of xnyzip_b200.verify (every input point against its cell's
    recovered point, the decoded cloud against those points)."""
    import numpy as np
    import torch
    from xnyzip_b200 import verify as V
    key = f"{workload}_{n}_seed{seed}"
    ref = load_digests().get(key)
    t0 = time.time()
    out = {"reference_digests": key if ref else None}
    if ref:
        out["input_matches_reference_input"] = V.sha256(host) == ref["input_sha256"]
    per, l2rep = {}, {}
    pts = d_pts.view(n, 3)
    for v in variants:
        q, l2, hil, rle = v
        name = vname(v)
        p, ln = ctx.compress_device(d_pts.data_ptr(), n, q, l2, hil, rle)
        torch.cuda.current_stream(dev).synchronize()
        got = {"container": V.sha256(V.device_view(p, (ln,), "|u1", dev))}
        dp, nout = ctx.decompress_device(p, ln, q, l2, rle)
        torch.cuda.current_stream(dev).synchronize()
        dec = V.device_view(dp, (nout, 3), "<f4", dev).clone()  # the context reuses its output buffer
        got["points"] = V.sha256(dec)
        got["frame"] = V.sha256(ctx.compress(d_pts, q, l2, hil, rle))
        if mono_frames is not None and v in mono_frames:
            got["e2e_frame"] = V.sha256(np.asarray(mono_frames[v]).tobytes())
            got["e2e_points"] = V.sha256(mono_outs[variants.index(v)])
        l2rep[name] = V.l2_report(ctx, pts, q, l2, decoded=dec)
        del dec
        if ref and name in ref["variants"]:
            r = ref["variants"][name]
            want = {"container": r["container_sha256"], "points": r["points_sha256"], "frame": r["frame_sha256"],
                    "e2e_frame": r["frame_sha256"], "e2e_points": r["points_sha256"]}
            checks = {k: got[k] == want[k] for k in got}
            per[name] = all(checks.values())
            if not per[name]:
                out.setdefault("failed_checks", {})[name] = [k for k, ok in checks.items() if not ok]
        else:
            per[name] = None
    torch.cuda.empty_cache()
    out["per_variant"] = per
    out["checked"] = ["container", "frame", "points", "e2e_frame", "e2e_points"] if mono_frames else \
        ["container", "frame", "points"]
    out["all_identical"] = bool(per) and all(x is True for x in per.values())
    out["l2"] = l2rep
    out["max_l2_error"] = max(r["max_l2_error"] for r in l2rep.values())
    out["over_bound"] = sum(r["over_bound"] for r in l2rep.values())
    out["decoded_mismatch_minus_z_minus1"] = sum(r["mismatch"] - r["z_minus1_points"] for r in l2rep.values())
    out["check_s"] = round(time.time() - t0, 1)
    return out


# ------------------------------------------------------------- learned block parameters ---
def learned_measure(ctx, stream, d_pts, n, variants, steps):
    """Extended container on the resident cloud: pre-zstd bits/point of the repos /
    SFC-delta stream's coding under each block mode (reference Huffman+GR container, one
    global parameter pair, the learned predictor, exhaustive search) and the device
    compress+decompress GB/s of each: the plain path (reference container), the learned
    predictor, the exhaustive per-block search it stands in for, and one global pair."""
    import torch
    import xnyzip_b200 as X
    modes = {"reference": 0, "global": 3, "learned": 2, "exhaustive": 1}
    out = {"bits_per_point_prezstd": {}, "block_stream_bits_per_value": {}, "fallback_fraction": {}}
    for v in variants:
        q, l2, hil, rle = v
        key = vname(v)
        bpp, bsv = {}, {}
        for name, m in modes.items():
            ctx.set_block_mode(m)
            _, ln = ctx.compress_device(d_pts.data_ptr(), n, q, l2, hil, rle)
            bpp[name] = round(8.0 * ln / n, 4)
            if m:
                bi = ctx.block_info()
                bsv[name] = round(bi["payload_bits"] / max(1, bi["values"]), 4)
                if name == "learned":
                    out["fallback_fraction"][key] = round(bi["fallback_blocks"] / max(1, bi["blocks"]), 5)
        ctx.set_block_mode(0)
        out["bits_per_point_prezstd"][key] = bpp
        out["block_stream_bits_per_value"][key] = bsv
    tot = {name: sum(v[name] for v in out["bits_per_point_prezstd"].values()) for name in modes}
    out["penalty_vs_exhaustive"] = round(tot["learned"] / tot["exhaustive"] - 1.0, 6)
    out["gain_vs_global"] = round(1.0 - tot["learned"] / tot["global"], 6)
    out["gain_vs_reference_container"] = round(1.0 - tot["learned"] / tot["reference"], 6)

    def step(mode):
        ctx.set_block_mode(mode)
        for q, l2, hil, rle in variants:
            p, ln = ctx.compress_device(d_pts.data_ptr(), n, q, l2, hil, rle)
            _, nout = ctx.decompress_device(p, ln, q, l2, rle)
            if nout != n:
                raise RuntimeError("learned round trip lost points")

    rates = {}
    for name, m in (("plain", 0), ("learned", 2), ("exhaustive", 1), ("global", 3)):
        step(m)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step(m)
        e1.record(stream)
        torch.cuda.synchronize()
        rates[name] = 12.0 * n * len(variants) * steps / (e0.elapsed_time(e1) / 1e3) / 1e9
    ctx.set_block_mode(0)
    out["device_GB_s"] = {k: round(v, 3) for k, v in rates.items()}
    out["speedup_vs_plain"] = round(rates["learned"] / rates["plain"], 4)
    out["speedup_vs_exhaustive"] = round(rates["learned"] / rates["exhaustive"], 4)
    out["note"] = ("extended container: the repos / SFC-delta stream in 1024-value blocks with per-block PFor "
                   "width and Golomb-Rice k; other streams as in the reference container; pre-zstd sizes")
    return out


# ------------------------------------------------------------------ the predictor's MLP ---
def mlp_measure(dev, stream, blocks=1 << 20, reps=10):
    """The block-parameter predictor's kernels alone: inference (xnyz_mlp_forward) and one
    training step's forward + backward (xnyz_mlp_train_batch) over `blocks` blocks of random
    features, CUDA events on `stream`, best of `reps`.  FLOPs per block: 2 * (34*64 + 64*64 +
    64*65) = 20,864 for inference (the dense layers), three times that for training (forward,
    dX and dW); reported against the measured dense bf16 peak as tensor-pipe context: the
    layers are 34-65 wide, far from a GEMM's shape."""
    import ctypes as C

    import numpy as np
    import torch
    from xnyzip_b200 import _native as N
    prm_host = np.fromfile(os.path.join(ROOT, "xnyzip_b200", "model", "blockparams.f32"), dtype=np.float32)
    prm = torch.from_numpy(prm_host).to(dev)
    g = torch.Generator(device=dev).manual_seed(5)
    feats = torch.rand((blocks, 34), generator=g, device=dev, dtype=torch.float32)
    feats[:, :32] /= feats[:, :32].sum(dim=1, keepdim=True)
    w = torch.randint(0, 33, (blocks,), generator=g, device=dev, dtype=torch.uint8)
    k = torch.randint(0, 32, (blocks,), generator=g, device=dev, dtype=torch.uint8)
    pw = torch.empty(blocks, dtype=torch.uint8, device=dev)
    pk = torch.empty_like(pw)
    grad = torch.zeros_like(prm)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    gather = torch.empty(N.mlp_gather_floats(blocks), dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    st = C.c_void_p(stream.cuda_stream)

    def fwd():
        N.check(N.mlp_forward(p(prm), p(feats), blocks, p(pw), p(pk), None, None, st))

    def train():
        N.check(N.mlp_train_batch(p(prm), p(feats), p(w), p(k), None, 0, blocks, 1.0 / blocks, p(grad), p(loss),
                                  p(gather), st))

    out = {}
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["bf16_tflops"])
    except Exception:
        peak = 1590.0
    for name, fn, flops in (("inference", fwd, 20864.0), ("training_step", train, 3 * 20864.0)):
        fn()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        t = min(ts)
        tf = flops * blocks / t / 1e12
        out[name] = {"ms": round(t * 1e3, 4), "blocks_per_s": round(blocks / t, 1), "TFLOP_s": round(tf, 3),
                     "frac_of_bf16_peak": round(tf / peak, 5)}
    out["blocks"] = blocks
    out["note"] = ("34-64-64-65 MLP, BF16 operands / FP32 accumulation on mma.sync m16n8k16; one inference "
                   "block = 1024 values of the repos / SFC-delta stream")
    del feats, grad, gather
    return out


# ------------------------------------------------------------------- the uneven batch ---
def batched_measure(ctx, stream, dev, count, workers):
    """Uneven batch (point counts log-uniform in [1e3, 4e6], terrain / clustered, bbox side
    log-uniform in [10, 1e4], L2 from {0.001, 0.01, 0.1}; TO, Hilbert, -rle), resident in HBM.
    plain: one context, per-cloud compress_device + decompress_device in order.  batched:
    xnyz_batch_roundtrip_device with worker streams per size class chosen by
    xnyz_batch_autotune; with the reference container and with learned block parameters.
    Device-synchronised wall clock (the work of one step spans many streams), best of 3."""
    import torch
    import xnyzip_b200 as X
    from xnyzip_b200 import synthetic_gpu as G
    t0 = time.time()
    clouds = G.batch_clouds(count, dev)
    torch.cuda.synchronize(dev)
    gen_s = time.time() - t0
    ptrs = [c.data_ptr() for c, _ in clouds]
    ns = [c.shape[0] for c, _ in clouds]
    params = [(1, l2, 1, 1, 1024) for _, l2 in clouds]
    total = float(sum(ns))

    def plain_step():
        for (c, l2), n in zip(clouds, ns):
            p, ln = ctx.compress_device(c.data_ptr(), n, 1, l2, True, True)
            _, nout = ctx.decompress_device(p, ln, 1, l2, True)
            if nout != n:
                raise RuntimeError("plain round trip lost points")

    rep_s, med_s = {}, {}

    def timed(fn, name, reps=3):
        """Best of `reps` timed runs after one warm-up (a run that grows a worker's workspace
        or loads its predictor pays cudaMalloc's device synchronisation)."""
        fn()
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            fn()
            torch.cuda.synchronize(dev)
            ts.append(time.perf_counter() - t)
        rep_s[name] = [round(x, 4) for x in ts]
        med_s[name] = statistics.median(ts)
        return min(ts)

    ctx.set_block_mode(0)
    t_plain = timed(plain_step, "plain")
    batch = X.Batch(0, workers)
    out = {"clouds": count, "points": int(total), "generate_s": round(gen_s, 2)}
    res = {"plain": t_plain}
    for name, mode in (("batched", 0), ("batched_learned", 2)):
        batch.set_block_mode(mode)
        tune = batch.autotune(ptrs, ns, params)

        def bstep():
            ln, no = batch.roundtrip_device(ptrs, ns, params)
            if list(no) != ns:
                raise RuntimeError("batched round trip lost points")
            return ln

        res[name] = timed(bstep, name)
        out[f"{name}_workers_per_class"] = tune
        out[f"{name}_bits_per_point_prezstd"] = round(8.0 * float(bstep().sum()) / total, 4)
    batch.close()
    out["rep_s"] = rep_s
    out["points_per_s"] = {k: round(total / v, 1) for k, v in res.items()}
    out["GB_s"] = {k: round(12.0 * total / v / 1e9, 3) for k, v in res.items()}
    out["speedup_vs_plain"] = {k: round(res["plain"] / v, 3) for k, v in res.items() if k != "plain"}
    out["GB_s_median"] = {k: round(12.0 * total / v / 1e9, 3) for k, v in med_s.items()}
    out["speedup_vs_plain_median"] = {k: round(med_s["plain"] / v, 3) for k, v in med_s.items() if k != "plain"}
    out["note"] = ("compress+decompress of every cloud, device-resident; size classes by point count "
                   "(powers of four from 16K), concurrent worker streams per class from the autotuner")
    del clouds
    torch.cuda.empty_cache()
    return out


# ------------------------------------------------------------- zstd frames on the GPU ---
def zstd_measure(ctx, stream, dev, points=4_000_000, piece=1 << 16, count=6360, reps=3):
    """xnyz_zstd_decompress_device on many small frames: the pre-zstd container of a
    `points`-point terrain cloud (TO, L2 0.01, Hilbert, -rle) cut into `piece`-byte pieces, each
    a libzstd 1.5.7 level-3 frame, repeated to `count` frames.  Device time with CUDA events on
    the context's stream (best of `reps`), the output compared bit for bit on the device; host
    libzstd (ZSTD_decompress) on the same frames with one thread and with every host thread."""
    import concurrent.futures as cf
    import ctypes as C

    import numpy as np
    import torch
    from xnyzip_b200 import _native as N
    z = C.CDLL(N.default_zstd_library())
    z.ZSTD_compressBound.restype = C.c_size_t
    z.ZSTD_compressBound.argtypes = [C.c_size_t]
    z.ZSTD_compress.restype = C.c_size_t
    z.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]
    z.ZSTD_decompress.restype = C.c_size_t
    z.ZSTD_decompress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]

    def frame(b):
        cap = z.ZSTD_compressBound(len(b))
        out = C.create_string_buffer(cap)
        size = z.ZSTD_compress(out, cap, b, len(b), 3)  # before reading out.raw, which copies
        return out.raw[:size]

    plain = ctx.compress(make_cloud("terrain", points, 7), 1, 0.01, True, True, use_zstd=False)
    pieces = [plain[i:i + piece] for i in range(0, len(plain), piece)]
    uniq = [frame(b) for b in pieces]
    k = -(-count // len(pieces))
    frames, content = (uniq * k)[:count], (pieces * k)[:count]
    caps = [len(b) for b in content]
    total = float(sum(caps))
    src = torch.frombuffer(bytearray(b"".join(frames)), dtype=torch.uint8).to(dev)
    ref = torch.frombuffer(bytearray(b"".join(content)), dtype=torch.uint8).to(dev)
    dst = torch.empty_like(ref)
    torch.cuda.synchronize(dev)  # the copies above ran on torch's stream, the decoder runs on the context's
    f_off = np.cumsum([0] + [len(f) for f in frames])[:-1]
    d_off = np.cumsum([0] + caps)[:-1]
    call = ([src.data_ptr() + int(o) for o in f_off], [len(f) for f in frames],
            [dst.data_ptr() + int(o) for o in d_off], caps)
    ctx.zstd_decompress_device(*call)  # sizes the workspace
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lens = ctx.zstd_decompress_device(*call)
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    exact = list(lens) == caps and bool(torch.equal(dst, ref))

    def host(idx):
        buf = C.create_string_buffer(piece)
        for i in idx:
            if z.ZSTD_decompress(buf, piece, frames[i], len(frames[i])) != caps[i]:
                raise RuntimeError("libzstd size mismatch")

    t = time.perf_counter()
    host(range(len(frames)))
    cpu1 = total / (time.perf_counter() - t)
    threads = os.cpu_count() or 1
    with cf.ThreadPoolExecutor(threads) as ex:
        t = time.perf_counter()
        list(ex.map(host, [range(j, len(frames), threads) for j in range(threads)]))
        cpun = total / (time.perf_counter() - t)
    del src, ref, dst
    torch.cuda.empty_cache()
    return {"frames": len(frames), "frame_content_bytes": piece, "content_bytes": int(total),
            "compressed_bytes": int(sum(len(f) for f in frames)), "gpu_GB_s": round(total / min(ts) / 1e9, 3),
            "gpu_ms": round(min(ts) * 1e3, 3), "rep_ms": [round(x * 1e3, 3) for x in ts], "bit_exact": exact,
            "host_libzstd_GB_s": {"1": round(cpu1 / 1e9, 3), str(threads): round(cpun / 1e9, 3)},
            "workload": f"pre-zstd container of a {points}-point terrain cloud (TO 0.01, Hilbert, -rle) in "
                        f"{piece}-byte pieces, each a libzstd level-3 frame, repeated to {count} frames; "
                        "one warp per frame"}


# ---------------------------------------------------------------------- CPU baselines ---
def _ref_lib():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, Reference, available_reference
    if available_reference():
        return Reference(), "reference"
    return Oracle(), "port"


def cpu_baseline(host, variants, sample_points, threads=1):
    """Reference CPU path on a bounded sample of the same cloud, one thread."""
    lib, kind = _ref_lib()
    x = host[:sample_points]
    tot_t = 0.0
    if kind == "reference":
        lib.quiet(True)
    try:
        for q, l2, hil, rle in variants:
            if kind == "reference":
                tc, td, _, _ = lib.roundtrip_timed(x, QNAME[q], l2, hil, rle)
            else:
                t0 = time.perf_counter()
                fr = lib.compress(x, QNAME[q], l2, hil, rle)
                t1 = time.perf_counter()
                lib.decompress(fr, QNAME[q], l2, rle)
                tc, td = t1 - t0, time.perf_counter() - t1
            tot_t += tc + td
    finally:
        if kind == "reference":
            lib.quiet(False)
    value = 12.0 * x.shape[0] * len(variants) / tot_t / 1e9
    return {"value": round(value, 5), "unit": "GB/s", "cores": threads, "kind": kind,
            "sample": f"first {x.shape[0]} points of the cloud, all {len(variants)} variants, compress+decompress "
                      f"timed by the reference's Timer ({tot_t:.1f} s)"}


def run_reference(args):
    """--impl reference: the reference CPU path on all host threads, in its per-chunk mode.

    The arm regenerates the bench's cloud (same generator, size and seed as the GPU arm's
    rank 0) and each step has every host thread compress and decompress, in all variants,
    its own --chunk-point chunk of it; the chunks are spread evenly over the cloud.  That is
    a bounded sample of the GPU arm's workload, whose config the line repeats unchanged."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    lib, kind = _ref_lib()
    threads = os.cpu_count() or 1
    chunk = args.chunk
    n = args.points or WORKLOADS[args.workload][1]
    host = make_cloud(args.workload, n, cloud_seed(args.workload, 0))
    stride = max(chunk, (n // threads) // chunk * chunk)
    starts = [min(t * stride, max(0, n - chunk)) for t in range(threads)]
    n_sample = sum(min(chunk, n - a) for a in starts)
    variants = WORKLOADS[args.workload][2][: args.variants]
    if kind == "reference":
        lib.quiet(True)

    def step():
        def work(t):
            x = host[starts[t]:starts[t] + chunk]
            for q, l2, hil, rle in variants:
                fr = lib.compress(x, QNAME[q], l2, hil, rle)
                lib.decompress(fr, QNAME[q], l2, rle)
        ths = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()

    try:
        for _ in range(args.warmup):
            step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        dt = time.perf_counter() - t0
    finally:
        if kind == "reference":
            lib.quiet(False)
    value = 12.0 * n_sample * len(variants) * args.steps / dt / 1e9
    sample = (f"{threads} host threads, each compressing and decompressing (all {len(variants)} variants, zstd "
              f"frames) one {chunk}-point chunk of the {n}-point cloud per step, chunks spread evenly over it "
              f"({n_sample} points per step; the reference's per-chunk mode)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.workload, n, variants, world),
        "sample": {"points_per_step": n_sample, "chunk_points": chunk, "threads": threads},
        "cpu_baseline": {"value": round(value, 5), "unit": "GB/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": round(value, 5), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="xnyz", choices=["xnyz", "reference"])
    ap.add_argument("--workload", default="terrain", choices=sorted(WORKLOADS))
    ap.add_argument("--points", type=int, default=0, help="points of the cloud (0: the workload's size)")
    ap.add_argument("--variants", type=int, default=6)
    ap.add_argument("--e2e-mode", default="roundtrip", choices=["roundtrip", "phases"],
                    help="e2e: xnyz_batch_roundtrip (each chunk compressed and decompressed on one worker) or "
                         "xnyz_batch_compress then xnyz_batch_decompress")
    ap.add_argument("--pipes", type=int, default=6, help="contexts (streams) the timed step spreads the variants over")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-points", type=int, default=1_000_000)
    ap.add_argument("--chunk", type=int, default=150_000, help="points per chunk (e2e and the reference arm)")
    ap.add_argument("--workers", type=int, default=0, help="batch worker threads (0: one per host thread)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-clouds", type=int, default=2048,
                    help="clouds of the uneven batch workload (0: skip that measurement)")
    ap.add_argument("--zstd-frames", type=int, default=6360,
                    help="frames of the GPU zstd decoding measurement (0: skip it)")
    ap.add_argument("--mlp-only", action="store_true",
                    help="run only the predictor's kernel measurement (inference and training) and print it")
    ap.add_argument("--zstd-only", action="store_true",
                    help="run only the GPU zstd decoding measurement and print it")
    ap.add_argument("--spheres", action=argparse.BooleanOptionalAction, default=True,
                    help="also measure the 175M-point spheres cloud (both variants, with parity) in its own sub-line")
    ap.add_argument("--parity", action=argparse.BooleanOptionalAction, default=True,
                    help="check the timed paths' outputs against the reference digests after the timed region")
    ap.add_argument("--learned", action=argparse.BooleanOptionalAction, default=True,
                    help="also measure the extended container with learned block parameters")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warning: fewer than 3 warm-up steps")
    if args.impl == "reference":
        run_reference(args)
    elif args.mlp_only:
        import torch
        stream = torch.cuda.Stream()
        print(json.dumps({"mlp_kernels": mlp_measure(torch.device("cuda", 0), stream)}), flush=True)
    elif args.zstd_only:
        import torch
        import xnyzip_b200 as X
        stream = torch.cuda.Stream()
        ctx = X.Context(0, stream=stream.cuda_stream)
        print(json.dumps({"zstd_frames": zstd_measure(ctx, stream, torch.device("cuda", 0),
                                                      count=args.zstd_frames or 6360)}), flush=True)
        ctx.close()
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
