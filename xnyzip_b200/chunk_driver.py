"""Per-chunk distributed driver: one process per GPU, torch.distributed for the host plumbing.

Restates the per-chunk mode of the reference's MPI driver (source/mpi_driver.cpp: arguments
:33-101, file layout :652-719, the per-block loop :809-941, the summary :945-1040):

* the input is a file of float32 x, y, z records; it is cut into blocks of `block_size`
  bytes (a multiple of 12; bytes past the last whole record are ignored), and rank r of N
  owns blocks r, r + N, r + 2N, ...;
* every block is compressed independently into its own zstd frame, byte-identical to a
  single-cloud compress of that block's points;
* rank r writes ``part_rank<rrrr>.bin`` (its frames in block order) and
  ``manifest_rank<rrrr>.jsonl`` (one record per block: block_id, input_offset, input_size,
  rank, part_offset, compressed_size); rank 0 writes ``summary.json`` (totals, per-rank
  figures, max-over-ranks phase times) and ``manifest_index.jsonl``.

GPU design: a rank reads a window of its blocks (bounded host memory) and compresses the
window as one batch through the library's batch entry points (worker threads with their own
contexts and streams on this rank's GPU), then appends the frames; nothing crosses ranks
but the final statistics, so there is no device collective (the reference's mapreduce mode,
which shuffles cells across ranks, is a different product and not built here).

`--shared-codebook` (-normal only): rank 0 fits complete Huffman codebooks on block 0
(fit_profile), broadcasts the profile, and every block is coded with it
(compress_with_profile), so that all frames carry the same codebook bytes.

`decompress` is the downstream tool the manifests are for: it rebuilds the point file with
every block's decoded points at the block's input offset (points inside a block in
container order, as the reference's decompressor returns them).

    torchrun --nproc-per-node 8 -m xnyzip_b200.chunk_driver compress --input pts.bin \\
        --output-dir out --block-size 67108860 --bound 0.01 --quantizer to --curve -h --mode -rle
    torchrun --nproc-per-node 8 -m xnyzip_b200.chunk_driver decompress --input-dir out \\
        --output pts.rec.bin --bound 0.01 --quantizer to --mode -rle
"""
from __future__ import annotations

import json
import os
import sys
import time
from dataclasses import dataclass, field

import numpy as np

POINT_BYTES = 12
# Quantizer codes as the reference driver's compress_block picks them (mpi_driver.cpp:129-130):
# "cube" is the cube quantizer and every other name, "adaptive" included, the truncated
# octahedron.
QUANTIZERS = {"cube": 0, "to": 1, "adaptive": 1}


@dataclass
class Args:
    input: str = ""
    output_dir: str = ""
    block_size: int = 64 * 1024 * 1024 - (64 * 1024 * 1024) % POINT_BYTES
    quantizer: str = "to"
    curve: str = "-z"
    mode: str = "-normal"
    bound: float = 1e-3
    direct_threshold: int = 1024
    verify_roundtrip: bool = False
    shared_codebook: bool = False
    window_bytes: int = 1 << 30  # host bytes of input per batch
    workers: int = 0


def _flags(argv, spec, prog):
    """`--key value` pairs (values may start with '-': "--curve -h", "--mode -rle") and
    boolean switches, as the reference's parse_args (mpi_driver.cpp:67-101)."""
    vals, i = {}, 0
    while i < len(argv):
        k = argv[i]
        if k in spec and spec[k] is bool:
            vals[k] = True
            i += 1
        elif k in spec:
            if i + 1 >= len(argv):
                raise SystemExit(f"{prog}: {k} needs a value")
            try:
                vals[k] = spec[k](argv[i + 1])
            except ValueError:
                raise SystemExit(f"{prog}: bad value for {k}: {argv[i + 1]}")
            i += 2
        else:
            raise SystemExit(f"{prog}: unknown argument {k}")
    return vals


def parse_compress_args(argv) -> Args:
    """The reference driver's flags (mpi_driver.cpp:67-101) plus --window-bytes / --workers."""
    spec = {"--input": str, "--output-dir": str, "--block-size": int, "--bound": float, "--quantizer": str,
            "--curve": str, "--mode": str, "--direct-threshold": int, "--shared-codebook": bool,
            "--verify-roundtrip": bool, "--window-bytes": int, "--workers": int}
    v = _flags(argv, spec, "chunk_driver compress")
    if "--input" not in v or "--output-dir" not in v:
        raise SystemExit("chunk_driver compress: --input and --output-dir are required")
    a = Args(input=v["--input"], output_dir=v["--output-dir"])
    a.block_size = v.get("--block-size", a.block_size)
    a.bound = v.get("--bound", a.bound)
    a.quantizer = v.get("--quantizer", a.quantizer)
    a.curve = v.get("--curve", a.curve)
    a.mode = v.get("--mode", a.mode)
    a.direct_threshold = v.get("--direct-threshold", a.direct_threshold)
    a.verify_roundtrip = v.get("--verify-roundtrip", False)
    a.shared_codebook = v.get("--shared-codebook", False)
    a.window_bytes = v.get("--window-bytes", a.window_bytes)
    a.workers = v.get("--workers", a.workers)
    if a.block_size <= 0 or a.block_size % POINT_BYTES:
        raise SystemExit("--block-size must be a positive multiple of 12")
    if a.quantizer not in QUANTIZERS:
        raise SystemExit("--quantizer must be cube, to or adaptive")
    if a.curve not in ("-z", "-h"):
        raise SystemExit("--curve must be -z or -h")
    if a.mode == "mapreduce":
        raise SystemExit("mapreduce mode (cross-rank cell shuffle) is not part of this driver")
    if a.mode not in ("-normal", "-rle"):
        raise SystemExit("--mode must be -normal or -rle")
    if a.shared_codebook and a.mode == "-rle":
        raise SystemExit("--shared-codebook is not implemented for -rle mode")
    return a


def parse_decompress_args(argv):
    spec = {"--input-dir": str, "--output": str, "--bound": float, "--quantizer": str, "--mode": str,
            "--workers": int}
    v = _flags(argv, spec, "chunk_driver decompress")
    if "--input-dir" not in v or "--output" not in v:
        raise SystemExit("chunk_driver decompress: --input-dir and --output are required")
    q, mode = v.get("--quantizer", "to"), v.get("--mode", "-normal")
    if q not in QUANTIZERS or mode not in ("-normal", "-rle"):
        raise SystemExit("chunk_driver decompress: bad --quantizer or --mode")
    return v["--input-dir"], v["--output"], q, v.get("--bound", 1e-3), mode, v.get("--workers", 0)


def block_layout(file_size: int, block_size: int):
    """(aligned_size, num_blocks) as mpi_driver.cpp:683-684."""
    aligned = file_size - file_size % POINT_BYTES
    return aligned, (aligned + block_size - 1) // block_size


def owned_blocks(num_blocks: int, rank: int, nranks: int):
    """Round-robin ownership (mpi_driver.cpp:819-820)."""
    return list(range(rank, num_blocks, nranks))


def block_extent(b: int, block_size: int, aligned: int):
    off = b * block_size
    return off, min(block_size, aligned - off)


def windows(blocks, block_size: int, window_bytes: int):
    """Consecutive groups of owned blocks holding at most window_bytes of input (>= 1 block)."""
    per = max(1, window_bytes // block_size)
    for i in range(0, len(blocks), per):
        yield blocks[i:i + per]


def part_name(rank: int) -> str:
    return f"part_rank{rank:04d}.bin"


def manifest_name(rank: int) -> str:
    return f"manifest_rank{rank:04d}.jsonl"


@dataclass
class RankStats:
    rank: int = 0
    input_bytes: int = 0
    compressed_bytes: int = 0
    blocks: int = 0
    read_s: float = 0.0
    comp_s: float = 0.0
    write_s: float = 0.0
    wall_s: float = 0.0
    warmup_s: float = 0.0
    records: list = field(default_factory=list)


class _Dist:
    """torch.distributed when launched by torchrun (gloo: only host-side statistics cross
    ranks), a single rank otherwise."""

    def __init__(self):
        self.rank = int(os.environ.get("RANK", "0"))
        self.size = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.pg = None
        if self.size > 1:
            import datetime

            import torch.distributed as dist
            if not dist.is_initialized():
                dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def broadcast(self, obj, src: int = 0):
        if not self.pg:
            return obj
        box = [obj]
        self.pg.broadcast_object_list(box, src=src)
        return box[0]

    def gather(self, obj):
        if not self.pg:
            return [obj]
        out = [None] * self.size
        self.pg.all_gather_object(out, obj)
        return out

    def close(self):
        if self.pg and self.pg.is_initialized():
            self.pg.destroy_process_group()


def _gpu_compressor(args: Args, device: int):
    """Batch compress of host clouds on this rank's GPU (the library's batch entry points)."""
    import xnyzip_b200 as X
    batch = X.Batch(device, args.workers)
    prm = (QUANTIZERS[args.quantizer], float(np.float32(args.bound)), args.curve == "-h", args.mode == "-rle",
           args.direct_threshold)

    def compress(clouds):
        return batch.compress(clouds, [prm] * len(clouds), use_zstd=True)

    compress.close = batch.close
    return compress


def _gpu_fit_profile(args: Args, device: int, pts: np.ndarray) -> bytes:
    """BlockCompressor::fit_profile on the warm-up block; the frame is dropped as there."""
    import xnyzip_b200 as X
    ctx = X.Context(device)
    try:
        _, prof = ctx.fit_profile(pts, QUANTIZERS[args.quantizer], float(np.float32(args.bound)), args.curve == "-h")
    finally:
        ctx.close()
    return prof


def _gpu_profile_compressor(args: Args, device: int, prof: bytes):
    """compress_with_profile of each block (mpi_driver.cpp:123-142), one context."""
    import xnyzip_b200 as X
    ctx = X.Context(device)
    q, l2, hil = QUANTIZERS[args.quantizer], float(np.float32(args.bound)), args.curve == "-h"

    def compress(clouds):
        return [ctx.compress_with_profile(c, q, l2, hil, prof) for c in clouds]

    compress.close = ctx.close
    return compress


def _verify_block(args: Args, ctx, pts: np.ndarray, frame: bytes, profile: bytes | None = None):
    """--verify-roundtrip (mpi_driver.cpp:838-899): decompress the frame and check every point
    against the input in container order; -rle blocks are skipped as there."""
    q = QUANTIZERS[args.quantizer]
    l2 = float(np.float32(args.bound))
    if profile is None:
        again, order = ctx.compress(pts, q, l2, args.curve == "-h", False, args.direct_threshold, use_zstd=True,
                                    want_order=True)
    else:
        again, order = ctx.compress_with_profile(pts, q, l2, args.curve == "-h", profile, want_order=True)
    if again != frame:
        raise RuntimeError("verify: recompressing the block gave different bytes")
    rec = ctx.decompress(frame, q, l2, False)
    if rec.shape != pts.shape:
        raise RuntimeError(f"verify: size mismatch (orig={pts.shape[0]} rec={rec.shape[0]})")
    err = np.linalg.norm(pts[order.astype(np.int64)] - rec, axis=1)
    over = int(np.count_nonzero(err > np.float32(args.bound)))
    if over:
        raise RuntimeError(f"verify: {over} points exceed the bound (max_err={float(err.max()):.6g})")
    return float(err.max()) if err.size else 0.0


def compress_file(args: Args, dist: _Dist, compressor=None, log=print) -> RankStats:
    """Runs the per-chunk compression of one rank.  `compressor(list of (n, 3) float32 arrays)
    -> list of frames` defaults to the GPU batch path on this rank's device; with
    --shared-codebook a given compressor is called as compressor(None, block 0's points) ->
    profile on rank 0 and as compressor(clouds, profile) -> frames."""
    os.makedirs(args.output_dir, exist_ok=True)
    file_size = os.path.getsize(args.input)
    aligned, num_blocks = block_layout(file_size, args.block_size)
    if num_blocks == 0:
        raise SystemExit("input has no whole point record")
    rank, nranks = dist.rank, dist.size
    mine = owned_blocks(num_blocks, rank, nranks)
    if rank == 0:
        log(f"input={args.input} size={file_size} aligned={aligned} block_size={args.block_size} "
            f"num_blocks={num_blocks} nranks={nranks}")
    own = compressor is None
    warmup_s = 0.0
    prof = None
    if args.shared_codebook:
        # rank 0 fits the codebooks on block 0 and every rank codes every block with them
        # (mpi_driver.cpp:722-781); a given `compressor(clouds, profile)` takes the profile
        dist.barrier()
        tw = time.perf_counter()
        if rank == 0:
            _, n0 = block_extent(0, args.block_size, aligned)
            warm = np.fromfile(args.input, dtype=np.float32, count=n0 // 4).reshape(-1, 3)
            prof = (_gpu_fit_profile(args, dist.local_rank, warm) if own else compressor(None, warm))
            log(f"[shared-codebook] rank 0 fit profile: blob={len(prof)} bytes")
        prof = dist.broadcast(prof, 0)
        dist.barrier()
        warmup_s = time.perf_counter() - tw
        if own:
            compressor = _gpu_profile_compressor(args, dist.local_rank, prof)
        else:
            compressor = (lambda clouds, _b=compressor, _p=prof: _b(clouds, _p))
    elif own:
        compressor = _gpu_compressor(args, dist.local_rank)
    ctx = None
    if args.verify_roundtrip and args.mode == "-normal":
        import xnyzip_b200 as X
        ctx = X.Context(dist.local_rank)
    elif args.verify_roundtrip and rank == 0:
        log("[verify] -rle mode: per-point roundtrip check skipped (RLE deduplicates)")
    st = RankStats(rank=rank)
    dist.barrier()
    t0 = time.perf_counter()
    with open(args.input, "rb") as fin, open(os.path.join(args.output_dir, part_name(rank)), "wb") as part, \
            open(os.path.join(args.output_dir, manifest_name(rank)), "w") as meta:
        for win in windows(mine, args.block_size, args.window_bytes):
            a = time.perf_counter()
            clouds, extents = [], []
            for b in win:
                off, nbytes = block_extent(b, args.block_size, aligned)
                fin.seek(off)
                raw = fin.read(nbytes)
                if len(raw) != nbytes:
                    raise RuntimeError(f"short read of block {b}")
                clouds.append(np.frombuffer(raw, dtype=np.float32).reshape(-1, 3))
                extents.append((b, off, nbytes))
            c = time.perf_counter()
            frames = compressor(clouds)
            if ctx is not None:
                for (b, _, _), pts, fr in zip(extents, clouds, frames):
                    _verify_block(args, ctx, pts, fr, prof if args.shared_codebook else None)
            w = time.perf_counter()
            for (b, off, nbytes), fr in zip(extents, frames):
                if fr is None:
                    raise RuntimeError(f"rank {rank} block {b}: compress failed")
                rec = {"block_id": b, "input_offset": off, "input_size": nbytes, "rank": rank,
                       "part_offset": part.tell(), "compressed_size": len(fr)}
                part.write(fr)
                meta.write(json.dumps(rec, separators=(",", ":")) + "\n")
                st.records.append(rec)
                st.input_bytes += nbytes
                st.compressed_bytes += len(fr)
                st.blocks += 1
            e = time.perf_counter()
            st.read_s += c - a
            st.comp_s += w - c
            st.write_s += e - w
            log(f"[progress] rank {rank}  blocks {st.blocks}/{len(mine)}  in={st.input_bytes / 1e6:.1f}MB "
                f"out={st.compressed_bytes / 1e6:.2f}MB  rank_elapsed={e - t0:.2f}s")
    if own:
        compressor.close()
    st.warmup_s = warmup_s
    if ctx is not None:
        ctx.close()
    dist.barrier()
    st.wall_s = time.perf_counter() - t0
    _write_summary(args, dist, st, num_blocks, log)
    dist.barrier()  # the summary and the manifest index exist when any rank returns
    return st


def _write_summary(args: Args, dist: _Dist, st: RankStats, num_blocks: int, log):
    """Totals and max-over-ranks phase times (mpi_driver.cpp:951-1036)."""
    mine = {k: getattr(st, k) for k in ("rank", "input_bytes", "compressed_bytes", "blocks", "read_s", "comp_s",
                                         "write_s", "wall_s", "warmup_s")}
    allr = dist.gather(mine)
    if dist.rank != 0:
        return
    g_in = sum(r["input_bytes"] for r in allr)
    g_out = sum(r["compressed_bytes"] for r in allr)
    wmax = max(r["wall_s"] for r in allr)
    wmin = min(r["wall_s"] for r in allr)
    summary = {
        "nranks": dist.size,
        "num_blocks": sum(r["blocks"] for r in allr),
        "block_size": args.block_size,
        "shared_codebook": bool(args.shared_codebook),
        "warmup_s": max(r["warmup_s"] for r in allr),
        "input_bytes": g_in,
        "compressed_bytes": g_out,
        "ratio": g_in / g_out if g_out else 0.0,
        "wall_max_s": wmax,
        "wall_min_s": wmin,
        "phase_max": {k: max(r[k + "_s"] for r in allr) for k in ("read", "comp", "write")},
        "end_to_end_throughput_GBps": g_in / wmax / 1e9 if wmax > 0 else 0.0,
        "per_rank": [{"rank": r["rank"], "input_bytes": r["input_bytes"], "compressed_bytes": r["compressed_bytes"],
                      "blocks": r["blocks"], "wall_s": r["wall_s"]} for r in allr],
    }
    with open(os.path.join(args.output_dir, "summary.json"), "w") as f:
        json.dump(summary, f, indent=2)
    with open(os.path.join(args.output_dir, "manifest_index.jsonl"), "w") as f:
        for r in range(dist.size):
            f.write(json.dumps({"rank": r, "part": part_name(r), "manifest": manifest_name(r)}) + "\n")
    log(f"\n=== run summary ===\nnranks={dist.size} num_blocks={summary['num_blocks']}\n"
        f"total_input_bytes={g_in} total_compressed_bytes={g_out} ratio={summary['ratio']:.4f}\n"
        f"wall_max_s={wmax:.4f} wall_min_s={wmin:.4f} load_balance={wmin / wmax if wmax else 0:.4f}\n"
        f"end_to_end_throughput={summary['end_to_end_throughput_GBps']:.4f} GB/s")


def read_manifests(input_dir: str):
    """All block records of a compressed directory, by block id."""
    recs = []
    with open(os.path.join(input_dir, "manifest_index.jsonl")) as f:
        index = [json.loads(line) for line in f if line.strip()]
    for ent in index:
        with open(os.path.join(input_dir, ent["manifest"])) as f:
            for line in f:
                if line.strip():
                    r = json.loads(line)
                    r["part"] = ent["part"]
                    recs.append(r)
    recs.sort(key=lambda r: r["block_id"])
    for i, r in enumerate(recs):
        if r["block_id"] != i:
            raise RuntimeError(f"manifests miss block {i}")
    return recs


def decompress_dir(input_dir: str, output: str, quantizer: str, bound: float, mode: str, dist: _Dist,
                   decompressor=None, workers: int = 0, window_bytes: int = 1 << 30, log=print):
    """Rebuilds the point file: block b's decoded points at its input offset.  Blocks are
    shared round-robin by block id; `decompressor(list of (frame, n_points)) -> list of
    (n, 3) float32 arrays` defaults to the GPU batch path."""
    recs = read_manifests(input_dir)
    total = recs[-1]["input_offset"] + recs[-1]["input_size"] if recs else 0
    if dist.rank == 0:
        with open(output, "wb") as f:
            f.truncate(total)
    dist.barrier()
    own = decompressor is None
    if own:
        import xnyzip_b200 as X
        batch = X.Batch(dist.local_rank, workers)
        prm = (QUANTIZERS[quantizer], float(np.float32(bound)), mode == "-rle")

        def decompressor(items):
            outs = [np.empty((n, 3), np.float32) for _, n in items]
            got = batch.decompress([fr for fr, _ in items], [prm] * len(items), outs)
            for o, g, (_, n) in zip(outs, got, items):
                if g != n:
                    raise RuntimeError(f"block decoded to {g} points, expected {n}")
            return outs
    mine = recs[dist.rank::dist.size]
    handles = {}
    done = 0
    with open(output, "r+b") as fout:
        per = max(1, window_bytes // max(1, max((r["input_size"] for r in recs), default=1)))
        for i in range(0, len(mine), per):
            win = mine[i:i + per]
            items = []
            for r in win:
                h = handles.get(r["part"])
                if h is None:
                    h = handles[r["part"]] = open(os.path.join(input_dir, r["part"]), "rb")
                h.seek(r["part_offset"])
                items.append((h.read(r["compressed_size"]), r["input_size"] // POINT_BYTES))
            pts = decompressor(items)
            for r, p in zip(win, pts):
                fout.seek(r["input_offset"])
                fout.write(np.ascontiguousarray(p, np.float32).tobytes())
                done += 1
    for h in handles.values():
        h.close()
    if own:
        batch.close()
    dist.barrier()
    if dist.rank == 0:
        log(f"decompressed {len(recs)} blocks into {output} ({total} bytes)")
    return done


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if not argv or argv[0] not in ("compress", "decompress"):
        raise SystemExit("usage: chunk_driver compress|decompress ...")
    if argv[0] == "compress":
        args = parse_compress_args(argv[1:])
    else:
        dargs = parse_decompress_args(argv[1:])
    dist = _Dist()
    try:
        if argv[0] == "compress":
            compress_file(args, dist)
        else:
            indir, out, q, bound, mode, workers = dargs
            decompress_dir(indir, out, q, bound, mode, dist, workers=workers)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
