"""Stage-level GPU parity through the C ABI (device pointers): quantize + shift, recover +
unshift, the Hilbert transform and the radix sort."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("quantizer", [0, 1])
@pytest.mark.parametrize("l2", [0.001, 0.05, 0.5])
def test_quantize_and_recover(ctx, oracle, quantizer, l2):
    from xnyzip_b200 import _native as N
    from xnyzip_b200 import synthetic as S
    x = np.concatenate([S.uniform(200_000, 1), S.planar(5000, 2), np.array([[0, 0, 0], [-0.0, 1, 2]], np.float32)])
    dx = torch.from_numpy(x).cuda()
    cells = torch.zeros((x.shape[0], 3), dtype=torch.int32, device="cuda")
    off = np.zeros(3, np.float32)
    N.check(N.stage_quantize(ctx.handle, _ptr(dx), x.shape[0], quantizer, l2, off.ctypes.data_as(C.c_void_p),
                             _ptr(cells)))
    ooff, oq = oracle.quantize(x, {0: "cube", 1: "to"}[quantizer], l2)
    assert off.tobytes() == ooff.tobytes()
    assert np.array_equal(cells.cpu().numpy(), oq)
    rec = torch.zeros_like(dx)
    N.check(N.stage_recover(ctx.handle, _ptr(cells), x.shape[0], quantizer, l2, off.ctypes.data_as(C.c_void_p),
                            _ptr(rec)))
    want = oracle.recover(oq, {0: "cube", 1: "to"}[quantizer], l2, ooff)
    assert rec.cpu().numpy().tobytes() == want.tobytes()


@pytest.mark.parametrize("inverse", [0, 1])
def test_hilbert_stage(ctx, oracle, inverse):
    from xnyzip_b200 import _native as N
    codes = np.arange(1 << 18, dtype=np.uint64)
    rng = np.random.default_rng(5)
    for it, c in [(20, codes)] + [(it, rng.integers(0, 2**63, 50_000, dtype=np.uint64)) for it in (1, 5, 10, 20)]:
        d = torch.from_numpy(c.view(np.int64)).cuda()
        o = torch.zeros_like(d)
        N.check(N.stage_hilbert(ctx.handle, _ptr(d), c.size, it, inverse, _ptr(o)))
        want = oracle.h2m(c, it) if inverse else oracle.m2h(c, it)
        assert np.array_equal(o.cpu().numpy().view(np.uint64), want), it


@pytest.mark.parametrize("n,bits", [(1, 64), (100, 8), (4096, 20), (4097, 33), (1_000_003, 42), (3_000_000, 64)])
def test_radix_sort_stage(ctx, n, bits):
    from xnyzip_b200 import _native as N
    rng = np.random.default_rng(n)
    hi = np.uint64((1 << bits) - 1) if bits < 64 else np.uint64(2**64 - 1)
    keys = rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    keys &= hi
    keys[: n // 3] = keys[0]  # many equal keys: stability matters
    payload = np.arange(n, dtype=np.uint32)
    dk = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    dv = torch.from_numpy(payload.view(np.int32).copy()).cuda()
    N.check(N.stage_sort(ctx.handle, _ptr(dk), _ptr(dv), n, bits))
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(dk.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), payload[order])
