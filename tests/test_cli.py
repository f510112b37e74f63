"""The XnYZip command line (xnyzip_b200/XnYZip) against the reference's own CLI built from its
sources (oracle/_ref/xnyzip_ref, source/main.cpp unmodified), with the same argv on the same
file: the decompressed output file, errors-<q>.bin of -normal runs, and the stdout lines the
reference's harnesses parse (main.cpp:15-203; chunk_sweep.py reads compression ratio and the
chunk byte counts).  Covers -rle / -normal, -z / -h, both quantizers, block and direct mode,
a forced block mode (threshold 0) and the chunk flags --offset / --count."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "xnyzip_b200", "XnYZip")
REF = os.path.join(ROOT, "oracle", "_ref", "xnyzip_ref")

# stdout lines both CLIs print (the reference's compressor also prints debug statistics -
# per-stream patch counts and entropies - which are not part of the command line contract)
KEYS = ("SFC type:", "Use RLE:", "Direct threshold:", "Chunk mode:", "Max L2 error:", "p2p psnr:", "MSE:",
        "Max diff:", "Unique points:", "Duplicate ratio:", "Encoding mode:", "compressed size of coords",
        "compression ratio of coords", "compression ratio:", "decompressed finished", "chunk input bytes:",
        "chunk compressed bytes:", "overflow count:")


def _contract_lines(out: str):
    return [ln.strip() for ln in out.splitlines() if ln.strip().startswith(KEYS)]


def _run(exe, workdir, args):
    os.makedirs(workdir, exist_ok=True)
    r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=600, cwd=workdir)
    assert r.returncode == 0, (exe, args, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    if not os.path.exists(REF):
        pytest.skip("the reference CLI was not built here (oracle/_ref)")
    if not os.path.exists(OURS):
        pytest.skip("xnyzip_b200/XnYZip is not built")
    from xnyzip_b200 import synthetic as S
    d = tmp_path_factory.mktemp("cli")
    S.terrain(40_000, 51, extent=300.0, amplitude=3.0, wavelength=150.0).tofile(d / "terrain.bin")
    np.random.default_rng(52).uniform(0, 3, (20_000, 3)).astype(np.float32).tofile(d / "small.bin")
    return d


# (input, [quantizer, L2, curve, mode], [direct threshold], [chunk flags])
CASES = [
    ("terrain.bin", ["to", "0.05", "-z", "-rle"], [], []),
    ("terrain.bin", ["cube", "0.01", "-h", "-normal"], [], []),
    ("terrain.bin", ["to", "0.05", "-h", "-normal"], ["0"], []),
    ("terrain.bin", ["to", "0.01", "-z", "-normal"], [], []),
    ("small.bin", ["to", "0.05", "-h", "-rle"], ["1024"], []),
    ("small.bin", ["cube", "0.05", "-z", "-normal"], [], []),
    ("terrain.bin", ["cube", "0.05", "-z", "-rle"], [], ["--offset=120000", "--count=180000"]),
    ("terrain.bin", ["to", "0.02", "-h", "-normal"], [], ["--offset=240000"]),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_cli_matches_reference(inputs, case):
    name, mode, threshold, flags = CASES[case]
    outs = {}
    for who, exe in (("ours", OURS), ("ref", REF)):
        wd = inputs / f"{who}_{case}"
        outs[who] = (_run(exe, str(wd), [str(inputs / name)] + mode + [str(wd / "decomp.bin")] + threshold + flags),
                     wd)
    (so, wo), (sr, wr) = outs["ours"], outs["ref"]
    assert (wo / "decomp.bin").read_bytes() == (wr / "decomp.bin").read_bytes()
    lo, lr = _contract_lines(so), _contract_lines(sr)
    assert lo == lr, "\n".join(f"{a!r} | {b!r}" for a, b in zip(lo, lr) if a != b) or (lo, lr)
    if "-normal" in mode:
        q = mode[0]
        eo = np.fromfile(wo / f"errors-{q}.bin", np.float32)
        er = np.fromfile(wr / f"errors-{q}.bin", np.float32)
        # position by position, up to points of one lattice cell taken in another order: where
        # the errors differ, the decoded point is that of a run of one cell
        assert eo.shape == er.shape and np.array_equal(np.sort(eo), np.sort(er))
        dec = np.fromfile(wo / "decomp.bin", np.float32).reshape(-1, 3)
        for i in np.flatnonzero(eo != er):
            assert (dec[i] == dec[max(i - 1, 0)]).all() or (dec[i] == dec[min(i + 1, len(dec) - 1)]).all(), i
    assert any(re.match(r"chunk compressed bytes:\s*(\d+)", ln) for ln in lr)
