"""GPU path against the reference's fixtures and the oracle: byte-identical zstd frames and
containers, bit-identical decoded points (integer / byte work: exact equality)."""
import hashlib
import os

import numpy as np
import pytest

from conftest import small_inputs

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.npz")
QN = {0: "cube", 1: "to", 2: "adaptive"}


def golden_names():
    return [str(n) for n in np.load(GOLDEN)["names"]]


@pytest.mark.parametrize("name", golden_names())
def test_gpu_matches_reference_fixture(ctx, name):
    f = np.load(GOLDEN)
    x = f[f"{name}/points"]
    q, hil, rle, th = (int(v) for v in f[f"{name}/params"])
    l2 = float(f[f"{name}/l2"][0])
    raw = ctx.compress(x, q, l2, hil, rle, th, use_zstd=False)
    assert raw == f[f"{name}/container"].tobytes()
    frame = ctx.compress(x, q, l2, hil, rle, th, use_zstd=True)
    assert frame == f[f"{name}/frame"].tobytes()
    # decode the reference's own frame
    dec = ctx.decompress(f[f"{name}/frame"].tobytes(), q, l2, rle)
    assert dec.tobytes() == f[f"{name}/decoded"].tobytes()


MODES = [(q, l2, hil, rle, th) for q in (0, 1, 2) for l2 in (0.05, 0.5) for hil in (0, 1) for rle in (0, 1)
         for th in (1024, 0)]


@pytest.mark.parametrize("kind", list(small_inputs(16).keys()))
def test_gpu_vs_oracle_matrix(ctx, oracle, kind):
    x = small_inputs(6000)[kind]
    for q, l2, hil, rle, th in MODES:
        want = oracle.compress(x, QN[q], l2, hil, rle, th, zstd=False)
        got = ctx.compress(x, q, l2, hil, rle, th, use_zstd=False)
        assert got == want, (kind, q, l2, hil, rle, th)
        dw = oracle.decompress(want, QN[q], l2, rle, zstd=False)
        dg = ctx.decompress(got, q, l2, rle, is_zstd=False)
        assert dg.tobytes() == dw.tobytes(), (kind, q, l2, hil, rle, th)


def test_gpu_config1_full(ctx):
    """Plain method, small: 1M uniform points, TO 0.05, -z, -rle (byte-identical frame)."""
    from xnyzip_b200 import synthetic as S
    f = np.load(GOLDEN)
    x = S.uniform(1_000_000, 0)
    frame = ctx.compress(x, 1, 0.05, 0, 1, 1024)
    assert len(frame) == int(f["config1/frame_len"][0])
    assert hashlib.sha256(frame).digest() == f["config1/frame_sha256"].tobytes()
    dec = ctx.decompress(frame, 1, 0.05, 1)
    assert hashlib.sha256(dec.tobytes()).digest() == f["config1/decoded_sha256"].tobytes()


@pytest.mark.parametrize("n", [1, 2, 3, 31, 4095, 4096, 4097, 70001])
def test_gpu_sizes_vs_oracle(ctx, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.uniform(0, 50, (n, 3)).astype(np.float32)
    for q, hil, rle in ((1, 1, 1), (0, 0, 0), (1, 0, 0)):
        want = oracle.compress(x, QN[q], 0.05, hil, rle, 1024, zstd=False)
        got = ctx.compress(x, q, 0.05, hil, rle, 1024, use_zstd=False)
        assert got == want
        assert ctx.decompress(got, q, 0.05, rle, is_zstd=False).tobytes() == \
            oracle.decompress(want, QN[q], 0.05, rle, zstd=False).tobytes()


def test_gpu_terrain_larger_vs_oracle(ctx, oracle):
    from xnyzip_b200 import synthetic as S
    x = S.terrain(600_000, 31, extent=2000.0, amplitude=10.0, wavelength=1000.0)
    for q, l2 in ((1, 0.01), (0, 0.1)):
        want = oracle.compress(x, QN[q], l2, 1, 1, 1024, zstd=False)
        got = ctx.compress(x, q, l2, 1, 1, 1024, use_zstd=False)
        assert got == want
        assert ctx.decompress(got, q, l2, 1, is_zstd=False).tobytes() == \
            oracle.decompress(want, QN[q], l2, 1, zstd=False).tobytes()


def test_gpu_normal_order_is_a_sort_permutation(ctx, oracle):
    """-normal reorders its input into container order (block_compressor.hpp:141-144)."""
    x = small_inputs(5000)["duplicates"]
    data, order = ctx.compress(x, 1, 0.05, 1, 0, 1024, use_zstd=False, want_order=True)
    assert sorted(order.tolist()) == list(range(x.shape[0]))
    _, oorder = oracle.compress(x, "to", 0.05, 1, 0, 1024, zstd=False, with_order=True)
    # equal cells may appear in any order; the cells in container order must agree
    oq = oracle.quantize(x, "to", 0.05)[1]
    assert np.array_equal(oq[order.astype(np.int64)], oq[oorder.astype(np.int64)])


def test_gpu_adaptive_zero_step_refused(ctx, xnyz):
    """A flat axis gets the step R * FLT_MIN / norm, which underflows to 0 when the cloud is
    large against the bound; the reference then casts NaN cells to INT_MIN and emits a
    container that does not decode to the input.  The GPU path refuses such clouds."""
    rng = np.random.default_rng(3)
    x = np.c_[rng.random((3000, 2)) * 1e6, np.full(3000, 7.5)].astype(np.float32)
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.compress(x, 2, 0.001, 1, 0)
    assert e.value.status == 6
    # a bound large enough keeps the step positive: flat axis at cell 0, exact round trip on z
    frame = ctx.compress(x, 2, 10.0, 1, 0)
    dec = ctx.decompress(frame, 2, 10.0, 0)
    assert np.all(dec[:, 2] == np.float32(7.5))
