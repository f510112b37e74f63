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
