"""Per-chunk driver on one GPU (world size 1): every block's frame is byte-identical to a
single-cloud compress of the block and to the oracle, --verify-roundtrip passes, and the
decompress tool rebuilds the file block by block."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("quantizer,curve,mode", [("to", "-h", "-rle"), ("cube", "-z", "-normal"),
                                                  ("adaptive", "-h", "-normal")])
def test_chunk_driver_gpu(tmp_path, ctx, oracle, quantizer, curve, mode):
    from xnyzip_b200 import chunk_driver as D
    from xnyzip_b200 import synthetic as S
    x = S.terrain(230_000, 12, extent=400.0, amplitude=4.0, wavelength=200.0)
    path = str(tmp_path / "pts.bin")
    x.tofile(path)
    outdir = str(tmp_path / "out")
    args = D.parse_compress_args(["--input", path, "--output-dir", outdir, "--block-size", str(12 * 50_000),
                                  "--bound", "0.02", "--quantizer", quantizer, "--curve", curve, "--mode", mode,
                                  "--window-bytes", str(12 * 120_000)] +
                                 # the reference's TO decoder misplaces cells quantized to z = -1 (its
                                 # driver's verify aborts there too): verify the cube runs only
                                 (["--verify-roundtrip"] if mode == "-normal" and quantizer == "cube" else []))
    st = D.compress_file(args, D._Dist(), log=lambda *a: None)
    assert st.blocks == 5
    q = D.QUANTIZERS[quantizer]
    l2 = float(np.float32(0.02))
    hil, rle = curve == "-h", mode == "-rle"
    recs = [json.loads(r) for r in open(os.path.join(outdir, D.manifest_name(0)))]
    part = open(os.path.join(outdir, D.part_name(0)), "rb").read()
    want_pts = []
    for r in recs:
        blk = x[r["input_offset"] // 12:(r["input_offset"] + r["input_size"]) // 12]
        fr = part[r["part_offset"]:r["part_offset"] + r["compressed_size"]]
        assert fr == ctx.compress(blk, q, l2, hil, rle, 1024), r["block_id"]
        if r["block_id"] == 0:  # the reference driver codes "adaptive" as "to"
            assert fr == oracle.compress(blk, {0: "cube", 1: "to"}[q], l2, hil, rle, 1024)
        want_pts.append(ctx.decompress(fr, q, l2, rle))
    rec_path = str(tmp_path / "rec.bin")
    D.decompress_dir(outdir, rec_path, quantizer, 0.02, mode, D._Dist(), log=lambda *a: None)
    got = np.fromfile(rec_path, np.float32).reshape(-1, 3)
    assert got.tobytes() == np.concatenate(want_pts).tobytes()
    summ = json.load(open(os.path.join(outdir, "summary.json")))
    assert summ["input_bytes"] == x.nbytes and summ["compressed_bytes"] == len(part)


def test_chunk_driver_gpu_shared_codebook(tmp_path, ctx, reference):
    """--shared-codebook: the profile fit on block 0 codes every block, byte-identical to the
    reference's compress_with_profile of each block."""
    from conftest import quiet_call
    from xnyzip_b200 import chunk_driver as D
    from xnyzip_b200 import synthetic as S
    x = S.terrain(160_000, 13, extent=400.0, amplitude=4.0, wavelength=200.0)
    path = str(tmp_path / "pts.bin")
    x.tofile(path)
    outdir = str(tmp_path / "out")
    args = D.parse_compress_args(["--input", path, "--output-dir", outdir, "--block-size", str(12 * 50_000),
                                  "--bound", "0.02", "--quantizer", "cube", "--curve", "-h", "--shared-codebook",
                                  "--verify-roundtrip"])
    st = D.compress_file(args, D._Dist(), log=lambda *a: None)
    assert st.blocks == 4
    l2 = float(np.float32(0.02))
    _, prof = ctx.fit_profile(x[:50_000], 0, l2, 1)
    assert prof == quiet_call(reference, reference.fit_profile, x[:50_000], "cube", l2, 1)[1]
    part = open(os.path.join(outdir, D.part_name(0)), "rb").read()
    for line in open(os.path.join(outdir, D.manifest_name(0))):
        r = json.loads(line)
        blk = x[r["input_offset"] // 12:(r["input_offset"] + r["input_size"]) // 12]
        fr = part[r["part_offset"]:r["part_offset"] + r["compressed_size"]]
        assert fr == quiet_call(reference, reference.compress_with_profile, blk, "cube", l2, 1, prof), r["block_id"]
    assert json.load(open(os.path.join(outdir, "summary.json")))["shared_codebook"] is True
