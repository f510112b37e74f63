"""The allocation-free sort entry point (xnyz_sort_noalloc).

It serves callers that cannot allocate device memory while they run, such as a real-time
loop that must not block on the CUDA allocator or a plugin whose host application owns all
device memory: the sort runs on a fixed scratch array in the library instead of a context
workspace.  The test calls it through the C ABI twice in a row and compares each result with
the context-based xnyz_stage_sort (integer keys: exact equality).  It sits in its own file,
collected last, and passes both alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(a, dtype):
    return torch.from_numpy(a.view(dtype).copy()).cuda()


def _keys(rng, n, bits):
    mask = np.uint64(2**64 - 1) if bits == 64 else np.uint64((1 << bits) - 1)
    keys = rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)
    keys &= mask
    keys[: n // 4] = keys[7]  # many equal keys: stability
    return keys


def test_sort_noalloc_matches_stage_sort(ctx):
    from xnyzip_b200 import _native as N
    rng = np.random.default_rng(2024)
    # calls in a row: an even pass count (42 bits: 6 passes), an odd one (20 bits: 3 passes, so
    # the result is copied back from the scratch array) and the size limit at 64 bits
    for n, bits in ((300_000, 42), (200_001, 20), (1 << 20, 64)):
        keys = _keys(rng, n, bits)
        payload = rng.permutation(n).astype(np.uint32)
        k_ref, v_ref = _dev(keys, np.int64), _dev(payload, np.int32)
        N.check(N.stage_sort(ctx.handle, C.c_void_p(k_ref.data_ptr()), C.c_void_p(v_ref.data_ptr()), n, bits))
        k_new, v_new = _dev(keys, np.int64), _dev(payload, np.int32)
        N.check(N.sort_noalloc(C.c_void_p(k_new.data_ptr()), C.c_void_p(v_new.data_ptr()), n, bits, None))
        assert torch.equal(k_new, k_ref)
        assert torch.equal(v_new, v_ref)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k_new.cpu().numpy().view(np.uint64), keys[order])
        assert np.array_equal(v_new.cpu().numpy().view(np.uint32), payload[order])


@pytest.mark.parametrize("n,bits", [(70_000, 20), (70_000, 33)])
def test_sort_noalloc_keys_only(ctx, n, bits):
    from xnyzip_b200 import _native as N
    keys = _keys(np.random.default_rng(n + bits), n, bits)
    k_ref = _dev(keys, np.int64)
    N.check(N.stage_sort(ctx.handle, C.c_void_p(k_ref.data_ptr()), None, n, bits))
    k_new = _dev(keys, np.int64)
    N.check(N.sort_noalloc(C.c_void_p(k_new.data_ptr()), None, n, bits, None))
    assert torch.equal(k_new, k_ref)
    assert np.array_equal(k_new.cpu().numpy().view(np.uint64), np.sort(keys, kind="stable"))


def test_sort_noalloc_rejects_oversize():
    from xnyzip_b200 import _native as N
    assert N.sort_noalloc(None, None, (1 << 20) + 1, 64, None) == 6  # XNYZ_ERR_UNSUPPORTED
