"""Batches of independent clouds (xnyz_batch_*): every frame and every decoded cloud equals
the per-cloud call's, whatever the worker count and order."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clouds():
    from xnyzip_b200 import synthetic as S
    rng = np.random.default_rng(11)
    clouds, params = [], []
    for i, n in enumerate([1, 7, 4096, 4097, 30000, 150000, 2500, 90001]):
        if i % 3 == 0:
            x = rng.uniform(0, 500, (n, 3)).astype(np.float32)
        elif i % 3 == 1:
            x = S.terrain(n, seed=100 + i)
        else:
            x = S.with_duplicates(n, seed=200 + i)
        clouds.append(x)
        params.append((i % 2, [0.001, 0.01, 0.1, 0.05][i % 4], i % 3 != 1, i % 4 != 3, [1024, 0, 4096][i % 3]))
    return clouds, params


@pytest.mark.parametrize("workers", [1, 3, 16])
def test_batch_matches_single_calls(ctx, xnyz, workers):
    clouds, params = _clouds()
    b = xnyz.Batch(0, workers)
    try:
        frames = b.compress(clouds, params)
        for x, p, f in zip(clouds, params, frames):
            assert f == ctx.compress(x, p[0], p[1], p[2], p[3], p[4])
        outs = [np.empty((x.shape[0] + 3, 3), np.float32) for x in clouds]
        ns = b.decompress(frames, [(p[0], p[1], p[3]) for p in params], outs)
        for x, p, f, o, n in zip(clouds, params, frames, outs, ns):
            ref = ctx.decompress(f, p[0], p[1], p[3])
            assert n == ref.shape[0]
            assert np.array_equal(o[:n].view(np.uint32), ref.view(np.uint32))
    finally:
        b.close()


@pytest.mark.parametrize("workers", [1, 4])
def test_batch_host_roundtrip_matches_single_calls(ctx, xnyz, workers):
    """xnyz_batch_roundtrip: the frames of xnyz_compress and the points of xnyz_decompress."""
    clouds, params = _clouds()
    b = xnyz.Batch(0, workers)
    try:
        outs = [np.full((x.shape[0], 3), np.nan, np.float32) for x in clouds]
        frames = b.roundtrip(clouds, params, outs, as_bytes=True)
        for x, p, f, o in zip(clouds, params, frames, outs):
            assert f == ctx.compress(x, p[0], p[1], p[2], p[3], p[4])
            ref = ctx.decompress(f, p[0], p[1], p[3])
            assert np.array_equal(o.view(np.uint32), ref.view(np.uint32))
    finally:
        b.close()


def test_batch_reports_failing_item(xnyz):
    clouds, params = _clouds()
    params = list(params)
    params[2] = (7, 0.01, 1, 1, 1024)  # unknown quantizer
    b = xnyz.Batch(0, 4)
    try:
        st = np.zeros(len(clouds), np.int64)
        with pytest.raises(xnyz.XnyzError) as e:
            b.compress(clouds, params, item_status=st)
        assert e.value.status == 1 and "cloud 2" in str(e.value)
        assert st[2] == 1 and st[[0, 1, 3, 4, 5, 6, 7]].sum() == 0
    finally:
        b.close()


def test_batch_roundtrip_device_and_autotune(xnyz, ctx):
    """Device round trip of an uneven batch on worker streams, by size class, with the
    autotuned worker counts: every container has the size of a lone compress_device call and
    decodes to all its points; also with learned block parameters."""
    import torch
    from xnyzip_b200 import synthetic as S
    sizes = [700, 5_000, 20_000, 70_000, 300_000, 1_100_000]
    clouds = [torch.from_numpy(S.terrain(n, 40 + i, extent=200.0 + 50 * i, amplitude=2.0, wavelength=90.0)).cuda()
              for i, n in enumerate(sizes)]
    params = [(1, (0.01, 0.05, 0.1)[i % 3], i % 2, 1, 1024) for i in range(len(sizes))]
    ptrs = [c.data_ptr() for c in clouds]
    b = xnyz.Batch(0, 4)
    one = xnyz.Context(0)  # a fresh context: the shipped predictor, like the batch's workers
    try:
        for mode in (0, 2):
            one.set_block_mode(mode)
            b.set_block_mode(mode)
            want = [one.compress_device(c.data_ptr(), n, q, l2, h, r, dt)[1]
                    for c, n, (q, l2, h, r, dt) in zip(clouds, sizes, params)]
            tune = b.autotune(ptrs, sizes, params)
            assert len(tune) == 6 and all(0 <= w <= 4 for w in tune)
            ln, no = b.roundtrip_device(ptrs, sizes, params)
            assert ln.tolist() == want
            assert no.tolist() == sizes
    finally:
        one.close()
        b.close()


def test_learned_mode_survives_workspace_growth_and_trim(xnyz):
    """The predictor's parameters live beside the context's workspace: growing the device
    container buffer (a larger cloud) or trimming the workspace must leave them in place, so a
    learned-mode compress after either writes the same container as before."""
    import torch
    from xnyzip_b200 import synthetic as S
    from xnyzip_b200 import verify as V
    small = torch.from_numpy(S.terrain(20_000, 61, extent=300.0, amplitude=2.0, wavelength=90.0)).cuda()
    large = torch.from_numpy(S.terrain(900_000, 62, extent=900.0, amplitude=2.0, wavelength=90.0)).cuda()
    c = xnyz.Context(0)
    try:
        c.set_block_mode(2)

        def digest(x):
            p, ln = c.compress_device(x.data_ptr(), x.shape[0], 1, 0.01, True, True)
            torch.cuda.synchronize()
            return ln, V.sha256(V.device_view(p, (ln,), "|u1", x.device))

        first = digest(small)
        digest(large)  # grows the device container buffer
        assert digest(small) == first
        from xnyzip_b200 import _native as N
        N.check(N.trim(c.handle))
        assert digest(small) == first
    finally:
        c.close()
