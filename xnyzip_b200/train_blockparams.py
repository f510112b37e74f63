"""Trains the block-parameter predictor of the extended container on the GPU.

    python -m xnyzip_b200.train_blockparams [--seeds 10-29] [--eval-seeds 1000-1004] [--epochs 6]

Data: clouds from the three generators of the plain-method workloads (uniform, terrain,
spheres; shapes as in xnyzip_b200.synthetic, drawn on the GPU with torch so that millions of
blocks take seconds), quantized with the plain method's parameter grid (to / cube, L2 bounds,
Morton / Hilbert, -rle / -normal).  For every cloud the library returns the repos /
SFC-delta stream (xnyz_stage_repos); per block of 1024 values the features
(xnyz_block_features) and the label, the exhaustive optimum (xnyz_block_search), are
computed on the device.

Training: the library's own kernels - forward, softmax cross-entropy of both heads and
backward on the tensor cores (xnyz_mlp_train_batch), Adam (xnyz_mlp_adam).  torch only holds
device memory and draws the random numbers.

Evaluation on held-out seeds: head accuracies and the size penalty of the predicted
parameters against the exhaustive optimum (with and without the low-confidence fallback).

Writes xnyzip_b200/model/blockparams.f32 (the FP32 parameters) and blockparams.json (the
report).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _torch():
    import torch
    return torch


from .synthetic_gpu import gen_spheres, gen_terrain, gen_uniform  # noqa: E402


def workloads(seed):
    """(generator, n, quantizer, l2, hilbert, rle) of one seed: the plain-method grid.  Point
    density shapes the deltas, so terrain alternates between 16M and 64M points (the
    terrain workload's size) and spheres between 16M and 48M."""
    out = [("uniform", 1_000_000, 1, 0.05, 0, 1)]
    nt = 64_000_000 if seed % 2 == 0 else 16_000_000
    ns = 48_000_000 if seed % 2 == 0 else 16_000_000
    for q in (1, 0):
        for l2 in (0.001, 0.01, 0.1):
            out.append(("terrain", nt, q, l2, 1, 1))
            out.append(("terrain", nt, q, l2, 0, 0))
    out.append(("spheres", ns, 1, 0.5, 0, 0))
    out.append(("spheres", ns, 1, 0.5, 0, 1))
    out.append(("spheres", ns, 0, 0.05, 1, 1))
    # small clouds fall into direct mode (the SFC-delta stream)
    out.append(("spheres_small", 400_000, 1, 0.1, 1, 1))
    out.append(("terrain_small", 400_000, 0, 0.1, 0, 1))
    return out


KIND_SALT = {"uniform": 1, "terrain": 2, "terrain_small": 3, "spheres": 4, "spheres_small": 5}


def make_cloud(kind, n, seed, dev):
    if kind == "uniform":
        return gen_uniform(n, seed, dev)
    if kind == "terrain":
        return gen_terrain(n, seed, dev)
    if kind == "terrain_small":
        return gen_terrain(n, seed, dev, extent=40.0, amplitude=0.5, wavelength=20.0)
    if kind == "spheres":
        return gen_spheres(n, seed, dev)
    if kind == "spheres_small":
        return gen_spheres(n, seed, dev, k=200, extent=60.0, r_median=5.0)
    raise ValueError(kind)


def collect(ctx, seeds, dev, keep_vals=True, log=print):
    """Device tensors: features [m, 34], w labels, k labels, exhaustive costs, and (keep_vals)
    the stream values themselves (for the size evaluation)."""
    torch = _torch()
    from . import _native as N
    feats, ws, ks, costs, vals = [], [], [], [], []
    t0 = time.time()
    for seed in seeds:
        for kind, n, q, l2, hil, rle in workloads(seed):
            pts = make_cloud(kind, n, seed * 1009 + KIND_SALT[kind], dev)
            buf = torch.empty(n, dtype=torch.int64, device=dev)
            cnt = ctx.stage_repos(pts.data_ptr(), n, q, l2, hil, rle, buf.data_ptr(), n)
            v = buf[:cnt]
            nb = (cnt + 1023) // 1024
            f = torch.empty((nb, 34), dtype=torch.float32, device=dev)
            w = torch.empty(nb, dtype=torch.uint8, device=dev)
            k = torch.empty(nb, dtype=torch.uint8, device=dev)
            c = torch.empty(nb, dtype=torch.int32, device=dev)
            s = torch.cuda.current_stream(dev).cuda_stream
            N.check(N.block_features(C.c_void_p(v.data_ptr()), cnt, C.c_void_p(f.data_ptr()), C.c_void_p(s)))
            N.check(N.block_search(C.c_void_p(v.data_ptr()), cnt, C.c_void_p(w.data_ptr()), C.c_void_p(k.data_ptr()),
                                   C.c_void_p(c.data_ptr()), C.c_void_p(s)))
            feats.append(f)
            ws.append(w)
            ks.append(k)
            costs.append(c)
            if keep_vals:
                vals.append(v.clone())
    torch.cuda.synchronize(dev)
    F = torch.cat(feats)
    log(f"collected {F.shape[0]} blocks from {len(seeds)} seeds in {time.time() - t0:.1f}s")
    return F, torch.cat(ws), torch.cat(ks), torch.cat(costs), vals


def init_params(seed=0):
    """He-initialised weights, zero biases, padding rows and columns zero."""
    rng = np.random.default_rng(seed)
    from . import _native as N
    n = N.model_param_count()
    p = np.zeros(n, np.float32)
    # W1 [64][48] (34 inputs used), b1, W2 [64][64], b2, W3 [72][64] (65 outputs used), b3
    o = 0
    for (rows, cols, used_c, used_r) in ((64, 48, 34, 64), (64, 64, 64, 64), (72, 64, 64, 65)):
        m = np.zeros((rows, cols), np.float32)
        m[:used_r, :used_c] = rng.normal(0.0, math.sqrt(2.0 / used_c), (used_r, used_c))
        p[o:o + rows * cols] = m.ravel()
        o += rows * cols + rows
    assert o == n
    return p


def train(F, W, K, epochs=6, batch=4096, lr=2e-3, seed=0, dev="cuda", log=print):
    torch = _torch()
    from . import _native as N
    m = F.shape[0]
    prm = torch.from_numpy(init_params(seed)).to(dev)
    grad = torch.zeros_like(prm)
    am = torch.zeros_like(prm)
    av = torch.zeros_like(prm)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    gather = torch.empty(N.mlp_gather_floats(batch), dtype=torch.float32, device=dev)
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    g = torch.Generator(device=dev).manual_seed(seed)
    steps = epochs * ((m + batch - 1) // batch)
    step = 0
    hist = []
    t0 = time.time()
    for ep in range(epochs):
        perm = torch.randperm(m, generator=g, device=dev).to(torch.int32)
        loss.zero_()
        for first in range(0, m, batch):
            cnt = min(batch, m - first)
            N.check(N.mlp_train_batch(C.c_void_p(prm.data_ptr()), C.c_void_p(F.data_ptr()), C.c_void_p(W.data_ptr()),
                                      C.c_void_p(K.data_ptr()), C.c_void_p(perm.data_ptr()), first, cnt,
                                      1.0 / cnt, C.c_void_p(grad.data_ptr()), C.c_void_p(loss.data_ptr()),
                                      C.c_void_p(gather.data_ptr()), s))
            step += 1
            lr_t = lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
            N.check(N.mlp_adam(C.c_void_p(prm.data_ptr()), C.c_void_p(grad.data_ptr()), C.c_void_p(am.data_ptr()),
                               C.c_void_p(av.data_ptr()), lr_t, step, s))
        torch.cuda.synchronize(dev)
        mean_loss = float(loss.item()) / ((m + batch - 1) // batch)
        hist.append(mean_loss)
        log(f"epoch {ep + 1}/{epochs}: mean loss {mean_loss:.4f} ({time.time() - t0:.1f}s)")
    return prm, hist, time.time() - t0


def evaluate(prm, F, W, K, Cst, vals, dev, fallback=0.5):
    """Accuracies and size penalties against the exhaustive optimum."""
    torch = _torch()
    from . import _native as N
    m = F.shape[0]
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    pw = torch.empty(m, dtype=torch.uint8, device=dev)
    pk = torch.empty(m, dtype=torch.uint8, device=dev)
    conf = torch.empty((m, 2), dtype=torch.float32, device=dev)
    N.check(N.mlp_forward(C.c_void_p(prm.data_ptr()), C.c_void_p(F.data_ptr()), m, C.c_void_p(pw.data_ptr()),
                          C.c_void_p(pk.data_ptr()), C.c_void_p(conf.data_ptr()), None, s))
    # predicted cost per block, stream by stream
    pc = torch.empty(m, dtype=torch.int32, device=dev)
    o = 0
    for v in vals:
        nb = (v.numel() + 1023) // 1024
        N.check(N.block_cost(C.c_void_p(v.data_ptr()), v.numel(), C.c_void_p(pw[o:o + nb].data_ptr()),
                             C.c_void_p(pk[o:o + nb].data_ptr()), C.c_void_p(pc[o:o + nb].data_ptr()), s))
        o += nb
    torch.cuda.synchronize(dev)
    low = conf.min(dim=1).values < fallback
    pcf = torch.where(low, Cst, pc)
    best = float(Cst.double().sum())
    return {
        "blocks": int(m),
        "acc_w": float((pw == W).float().mean()),
        "acc_k": float((pk == K).float().mean()),
        "acc_both": float(((pw == W) & (pk == K)).float().mean()),
        "penalty": float(pc.double().sum()) / best - 1.0,
        "penalty_with_fallback": float(pcf.double().sum()) / best - 1.0,
        "fallback_fraction": float(low.float().mean()),
        "fallback_confidence": fallback,
    }


def evaluate_acc(prm, F, W, K, dev):
    torch = _torch()
    from . import _native as N
    m = F.shape[0]
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    pw = torch.empty(m, dtype=torch.uint8, device=dev)
    pk = torch.empty(m, dtype=torch.uint8, device=dev)
    N.check(N.mlp_forward(C.c_void_p(prm.data_ptr()), C.c_void_p(F.data_ptr()), m, C.c_void_p(pw.data_ptr()),
                          C.c_void_p(pk.data_ptr()), None, None, s))
    torch.cuda.synchronize(dev)
    return {"acc_w": float((pw == W).float().mean()), "acc_k": float((pk == K).float().mean())}


def _seeds(spec):
    a, b = spec.split("-")
    return list(range(int(a), int(b) + 1))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", default="10-29")
    ap.add_argument("--eval-seeds", default="1000-1004")
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--fallback", type=float, default=0.5)
    ap.add_argument("--out", default=os.path.join(HERE, "model", "blockparams"))
    a = ap.parse_args(argv)
    torch = _torch()
    from . import Context
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    # one stream for torch's generators and the library (the legacy default stream does not
    # order against the library's own non-blocking stream)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx = Context(0, stream=stream.cuda_stream)
    F, W, K, Cst, _ = collect(ctx, _seeds(a.seeds), dev, keep_vals=False)
    Fe, We, Ke, Ce, ve = collect(ctx, _seeds(a.eval_seeds), dev)
    prm, hist, secs = train(F, W, K, a.epochs, a.batch, a.lr, dev=dev)
    rep = {"held_out": evaluate(prm, Fe, We, Ke, Ce, ve, dev, a.fallback),
           "held_out_by_threshold": {str(t): evaluate(prm, Fe, We, Ke, Ce, ve, dev, t)
                                     for t in (0.0, 0.3, 0.5, 0.7, 0.9)},
           "train_accuracy": {k: v for k, v in evaluate_acc(prm, F, W, K, dev).items()},
           "train_blocks": int(F.shape[0]), "eval_blocks": int(Fe.shape[0]), "epochs": a.epochs,
           "batch": a.batch, "lr": a.lr, "loss_per_epoch": hist, "train_seconds": round(secs, 2),
           "seeds": a.seeds, "eval_seeds": a.eval_seeds}
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    prm.cpu().numpy().astype(np.float32).tofile(a.out + ".f32")
    with open(a.out + ".json", "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps(rep))
    ctx.close()


if __name__ == "__main__":
    main()
