"""Host-side parts of the product, no GPU: the library loads and exports the C ABI, and the
Hilbert tables and Huffman codebook replay match the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(xnyz):
    from xnyzip_b200 import _native as N
    header = open(os.path.join(ROOT, "include", "xnyz.h")).read()
    declared = sorted(set(re.findall(r"\b(xnyz_[a-z_0-9]+)\s*\(", header)))
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(N.lib, name), name
    assert sorted(N.EXPORTED) == declared


def test_context_without_gpu_reports_status(xnyz):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(xnyz.XnyzError) as e:
        xnyz.Context(0)
    assert e.value.status == 8


def _host_hilbert(codes, it, inverse):
    from xnyzip_b200 import _native as N
    c = np.ascontiguousarray(codes, dtype=np.uint64)
    o = np.zeros_like(c)
    N.check(N.host_hilbert(c.ctypes.data_as(C.c_void_p), c.size, it, int(inverse), o.ctypes.data_as(C.c_void_p)))
    return o


def test_hilbert_tables_match_oracle(xnyz, oracle):
    codes = np.arange(1 << 18, dtype=np.uint64)
    assert np.array_equal(_host_hilbert(codes, 20, 0), oracle.m2h(codes, 20))
    assert np.array_equal(_host_hilbert(codes, 20, 1), oracle.h2m(codes, 20))
    rng = np.random.default_rng(1)
    for it in range(1, 21):
        c = rng.integers(0, 2**63, 3000, dtype=np.uint64) | (rng.integers(0, 2, 3000, dtype=np.uint64) << np.uint64(63))
        assert np.array_equal(_host_hilbert(c, it, 0), oracle.m2h(c, it)), it
        assert np.array_equal(_host_hilbert(c, it, 1), oracle.h2m(c, it)), it


def _codebook(data, kind, count_stream=False):
    """Statistics the kernels produce (frequency + first occurrence) -> host codebook."""
    from xnyzip_b200 import _native as N
    d = np.asarray(data)
    vals, first, counts = np.unique(d, return_index=True, return_counts=True)
    sym = vals.astype(np.int64).astype(np.uint64)
    first = first.astype(np.uint64)
    counts = counts.astype(np.uint64)
    meta = np.zeros(1 << 20, np.uint8)
    ml = C.c_uint64(meta.size)
    bits = C.c_uint64()
    eg = C.c_int()
    N.check(N.host_codebook(kind, int(count_stream), sym.ctypes.data_as(C.c_void_p), counts.ctypes.data_as(C.c_void_p),
                            first.ctypes.data_as(C.c_void_p), sym.size, d.size, meta.ctypes.data_as(C.c_void_p),
                            C.byref(ml), C.byref(bits), C.byref(eg)))
    return meta[: ml.value].tobytes(), bits.value, bool(eg.value)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_codebook_replay_matches_oracle_meta(xnyz, oracle, kind):
    rng = np.random.default_rng(10 + kind)
    cases = {
        0: [rng.integers(0, 256, 20000), (rng.geometric(0.2, 20000) % 256), np.zeros(64), np.array([5]),
            np.concatenate([np.zeros(1000), np.arange(1, 256)])],
        1: [rng.integers(1, 9, 20000), np.full(9, 4), rng.integers(1, 3, 1001)],
        2: [rng.geometric(0.6, 30000), np.ones(500), rng.integers(1, 40, 9000)],
    }[kind]
    for d in cases:
        meta, bits, eg = _codebook(d, kind)
        ometa, oenc = oracle.huffman(d, kind)
        assert meta == ometa
        assert (bits + 7) // 8 == len(oenc)


def test_count_stream_codebook_matches_oracle_container(xnyz, oracle):
    """The -rle count stream: build, measure, maybe switch to exp-Golomb, rebuild."""
    rng = np.random.default_rng(4)
    for reps in (rng.integers(1, 3, 2000), rng.integers(1, 400, 300), np.ones(50, np.int64)):
        base = rng.uniform(0, 100, (reps.size, 3)).astype(np.float32)
        x = np.repeat(base, reps, axis=0)
        raw = oracle.compress(x, "to", 0.001, 1, 1, 1024, zstd=False)
        # The exp-Golomb decision depends on the count multiset only, not on its order.
        _, _, eg = _codebook(reps, 2, count_stream=True)
        assert (b"\xe1\xc1\x01\x01" in raw) == eg


UDIV_CHECK = r"""
#include "kernels.h"
#include <cstdio>
#include <random>
using u64 = unsigned long long;
// the device formula of k_decode.cu's udiv, with a 128-bit product for mulhi
static u64 udiv(u64 x, const xnyz::dev::U64Div& d) {
    const u64 t = (u64)(((unsigned __int128)d.m * x) >> 64);
    return (t + ((x - t) >> d.sh1)) >> d.sh2;
}
int main() {
    std::mt19937_64 rng(7);
    u64 ds[] = {1, 2, 3, 5, 7, 64, 127, 128, 129, 1000, 78126, (1ull << 21) + 1, (1ull << 31) - 1, 1ull << 31,
                (1ull << 32) - 5, 0xffffffffull, 1ull << 40, (1ull << 63) + 3, ~0ull};
    long bad = 0, checks = 0;
    for (u64 d : ds) {
        const auto m = xnyz::dev::make_u64div(d);
        u64 xs[] = {0, 1, d - 1, d, d + 1, 2 * d - 1, ~0ull, ~0ull - 1, 1ull << 63, (1ull << 58) * 3 + 11};
        for (u64 x : xs) { ++checks; if (udiv(x, m) != x / d) ++bad; }
        for (int i = 0; i < 200000; ++i) {
            const u64 x = rng() >> (rng() % 64);
            ++checks;
            if (udiv(x, m) != x / d) ++bad;
        }
    }
    std::printf("%ld %ld\n", checks, bad);
    return bad != 0;
}
"""


def test_invariant_divisor_multiply(tmp_path):
    """The block-coordinate division of recover_units (x / nx, x / ny for any u64 block id,
    wrapped ids of the z = -1 cells included) by a precomputed multiplier equals x / d."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    src = tmp_path / "udiv.cpp"
    src.write_text(UDIV_CHECK)
    exe = tmp_path / "udiv"
    csrc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "xnyzip_b200", "csrc")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", csrc, str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout
