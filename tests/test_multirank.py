"""Multi-rank host logic on CPU (gloo, world size 2): the per-chunk driver's block ownership,
part files, manifests, summary and reassembly, with a stand-in codec (the GPU codec is
covered by tests/test_gpu_chunk_driver.py), and the bench's max-over-ranks timing."""
import json
import os
import socket
import zlib

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))


def _fake_compress(clouds):
    return [zlib.compress(np.ascontiguousarray(c, np.float32).tobytes()) for c in clouds]


def _fake_decompress(items):
    return [np.frombuffer(zlib.decompress(fr), np.float32).reshape(-1, 3) for fr, _ in items]


def _driver_worker(rank, world, port, path, outdir, recpath):
    _env(rank, world, port)
    from xnyzip_b200 import chunk_driver as D
    dist = D._Dist()
    try:
        args = D.Args(input=path, output_dir=outdir, block_size=12 * 1000, window_bytes=12 * 2500)
        D.compress_file(args, dist, compressor=_fake_compress, log=lambda *a: None)
        D.decompress_dir(outdir, recpath, "to", 0.01, "-normal", dist, decompressor=_fake_decompress,
                         window_bytes=12 * 1500, log=lambda *a: None)
    finally:
        dist.close()


def test_chunk_driver_two_ranks(tmp_path):
    from xnyzip_b200 import chunk_driver as D
    rng = np.random.default_rng(4)
    data = rng.random(10_500 * 3, dtype=np.float32).tobytes() + b"\x01\x02\x03\x04\x05\x06\x07"
    path = str(tmp_path / "pts.bin")
    with open(path, "wb") as f:
        f.write(data)
    outdir = str(tmp_path / "out")
    recpath = str(tmp_path / "rec.bin")
    mp.start_processes(_driver_worker, args=(2, _free_port(), path, outdir, recpath), nprocs=2, join=True,
                       start_method="spawn")

    aligned, nblocks = D.block_layout(len(data), 12 * 1000)
    assert (aligned, nblocks) == (126_000, 11)
    for r in (0, 1):
        recs = [json.loads(x) for x in open(os.path.join(outdir, D.manifest_name(r)))]
        assert [x["block_id"] for x in recs] == list(range(r, 11, 2))
        part = open(os.path.join(outdir, D.part_name(r)), "rb").read()
        pos = 0
        for x in recs:
            assert x["rank"] == r and x["part_offset"] == pos
            assert x["input_offset"] == 12_000 * x["block_id"]
            assert x["input_size"] == min(12_000, aligned - x["input_offset"])
            fr = part[pos:pos + x["compressed_size"]]
            assert zlib.decompress(fr) == data[x["input_offset"]:x["input_offset"] + x["input_size"]]
            pos += x["compressed_size"]
        assert pos == len(part)
    summ = json.load(open(os.path.join(outdir, "summary.json")))
    assert summ["nranks"] == 2 and summ["num_blocks"] == 11 and summ["input_bytes"] == aligned
    assert [p["blocks"] for p in summ["per_rank"]] == [6, 5]
    assert summ["wall_max_s"] >= summ["wall_min_s"] > 0
    assert summ["wall_max_s"] == max(p["wall_s"] for p in summ["per_rank"])
    idx = [json.loads(x) for x in open(os.path.join(outdir, "manifest_index.jsonl"))]
    assert [i["part"] for i in idx] == [D.part_name(0), D.part_name(1)]
    assert open(recpath, "rb").read() == data[:aligned]


def test_chunk_driver_flags():
    from xnyzip_b200 import chunk_driver as D
    with pytest.raises(SystemExit):
        D.parse_compress_args(["--input", "x", "--output-dir", "o", "--block-size", "100"])
    with pytest.raises(SystemExit):
        D.parse_compress_args(["--input", "x", "--output-dir", "o", "--mode", "mapreduce"])
    with pytest.raises(SystemExit):
        D.parse_compress_args(["--input", "x", "--output-dir", "o", "--shared-codebook", "--mode", "-rle"])
    assert D.parse_compress_args(["--input", "x", "--output-dir", "o", "--shared-codebook"]).shared_codebook
    assert D.QUANTIZERS["adaptive"] == D.QUANTIZERS["to"] == 1  # as the reference driver's compress_block
    a = D.parse_compress_args(["--input", "x", "--output-dir", "o", "--block-size", "120", "--quantizer", "adaptive",
                               "--curve", "-h", "--mode", "-rle", "--bound", "0.5"])
    assert (a.block_size, a.quantizer, a.curve, a.mode, a.bound) == (120, "adaptive", "-h", "-rle", 0.5)
    assert D.owned_blocks(7, 1, 3) == [1, 4]
    assert list(D.windows([0, 2, 4, 6, 8], 100, 250)) == [[0, 2], [4, 6], [8]]
    assert list(D.windows([1], 100, 10)) == [[1]]


def _sync_worker(rank, world, port, q):
    _env(rank, world, port)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        s = bench.RankSync(world)
        s.barrier()
        q.put((rank, s.max(1.5 + rank)))
    finally:
        dist.destroy_process_group()


def test_bench_max_over_ranks():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    mp.start_processes(_sync_worker, args=(2, _free_port(), q), nprocs=2, join=True, start_method="spawn")
    got = sorted(q.get() for _ in range(2))
    assert got == [(0, 2.5), (1, 2.5)]


def _fake_profile_compress(clouds, prof):
    if clouds is None:  # the fit on block 0: a profile that names the block's bytes
        return b"P" + zlib.compress(np.ascontiguousarray(prof, np.float32).tobytes())[:16]
    return [prof + zlib.compress(np.ascontiguousarray(c, np.float32).tobytes()) for c in clouds]


def _shared_worker(rank, world, port, path, outdir):
    _env(rank, world, port)
    from xnyzip_b200 import chunk_driver as D
    dist = D._Dist()
    try:
        args = D.parse_compress_args(["--input", path, "--output-dir", outdir, "--block-size", str(12 * 700),
                                      "--shared-codebook"])
        D.compress_file(args, dist, compressor=_fake_profile_compress, log=lambda *a: None)
    finally:
        dist.close()


def test_chunk_driver_shared_codebook_two_ranks(tmp_path):
    """Every block of every rank is coded with the profile rank 0 fit on block 0."""
    from xnyzip_b200 import chunk_driver as D
    x = np.random.default_rng(8).random((5000, 3), dtype=np.float32)
    path = str(tmp_path / "pts.bin")
    x.tofile(path)
    outdir = str(tmp_path / "out")
    mp.start_processes(_shared_worker, args=(2, _free_port(), path, outdir), nprocs=2, join=True,
                       start_method="spawn")
    want = _fake_profile_compress(None, x[:700])
    seen = 0
    for r in (0, 1):
        part = open(os.path.join(outdir, D.part_name(r)), "rb").read()
        for line in open(os.path.join(outdir, D.manifest_name(r))):
            rec = json.loads(line)
            fr = part[rec["part_offset"]:rec["part_offset"] + rec["compressed_size"]]
            assert fr.startswith(want)
            seen += 1
    assert seen == 8
    summ = json.load(open(os.path.join(outdir, "summary.json")))
    assert summ["shared_codebook"] is True and summ["warmup_s"] > 0
