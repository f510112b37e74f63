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
                                 (["--verify-roundtrip"] if mode == "-normal" else []))
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
        if r["block_id"] == 0:
            assert fr == oracle.compress(blk, quantizer, l2, hil, rle, 1024)
        want_pts.append(ctx.decompress(fr, q, l2, rle))
    rec_path = str(tmp_path / "rec.bin")
    D.decompress_dir(outdir, rec_path, quantizer, 0.02, mode, D._Dist(), log=lambda *a: None)
    got = np.fromfile(rec_path, np.float32).reshape(-1, 3)
    assert got.tobytes() == np.concatenate(want_pts).tobytes()
    summ = json.load(open(os.path.join(outdir, "summary.json")))
    assert summ["input_bytes"] == x.nbytes and summ["compressed_bytes"] == len(part)
