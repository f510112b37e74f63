"""Failure handling without faulting the GPU: corrupted or truncated containers and bad
arguments come back as status codes, and the context keeps working afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _good(ctx):
    x = np.random.default_rng(1).uniform(0, 100, (20000, 3)).astype(np.float32)
    return x, ctx.compress(x, 1, 0.05, 1, 1, 1024, use_zstd=False)


def test_truncated_containers_fail_cleanly(ctx, xnyz):
    x, raw = _good(ctx)
    for cut in (0, 5, 16, 40, len(raw) // 3, len(raw) // 2, len(raw) - 13, len(raw) - 1):
        with pytest.raises(xnyz.XnyzError) as e:
            ctx.decompress(raw[:cut], 1, 0.05, 1, is_zstd=False)
        assert e.value.status in (2, 6)
    # still usable
    assert ctx.decompress(raw, 1, 0.05, 1, is_zstd=False).shape == (20000, 3)


def test_corrupted_payload_never_traps(ctx, xnyz):
    x, raw = _good(ctx)
    rng = np.random.default_rng(7)
    for trial in range(40):
        b = bytearray(raw)
        for _ in range(1 + trial % 5):
            i = int(rng.integers(38, len(b) - 12))
            b[i] ^= 1 << int(rng.integers(0, 8))
        try:
            ctx.decompress(bytes(b), 1, 0.05, 1, is_zstd=False)
        except xnyz.XnyzError as e:
            assert e.status in (2, 4, 6)
    assert ctx.decompress(raw, 1, 0.05, 1, is_zstd=False).shape == (20000, 3)


def test_bad_arguments(ctx, xnyz):
    x = np.zeros((10, 3), np.float32)
    with pytest.raises(xnyz.XnyzError):
        ctx.compress(x, 7, 0.05, 0, 0)
    with pytest.raises(xnyz.XnyzError):
        ctx.compress(x, 1, -1.0, 0, 0)
    with pytest.raises(xnyz.XnyzError):
        ctx.compress(np.zeros((0, 3), np.float32), 1, 0.05, 0, 0)
    bad = x.copy()
    bad[3, 1] = np.nan
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.compress(bad, 1, 0.05, 0, 0)
    assert e.value.status == 6
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.decompress(b"not a zstd frame", 1, 0.05, 1)
    assert e.value.status == 7
