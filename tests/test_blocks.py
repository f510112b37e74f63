"""Extended container: block-parameter coder and its predictor.

CPU tests pin the numpy restatement (oracle/blocks_oracle.py): the exhaustive search against
the full cost table, encode -> decode round trips, and the predictor's analytic gradient
against finite differences.  GPU tests check the kernels through the C ABI against it:
features, search, costs, the block stream's bytes, MLP logits and gradients, and that the
extended container decodes to exactly the points of the reference container.
"""
import ctypes as C
import os

import numpy as np
import pytest

import blocks_oracle as B

HERE = os.path.dirname(os.path.abspath(__file__))


def streams():
    """Seeded repos-like streams: geometric values, zeros, runs, huge escapes, ragged tails."""
    rng = np.random.default_rng(11)
    out = {}
    out["geometric"] = rng.geometric(0.02, 5000).astype(np.uint64)
    v = rng.geometric(0.3, 4100).astype(np.uint64) - np.uint64(1)
    v[::97] = rng.integers(1 << 20, 1 << 40, v[::97].size, dtype=np.uint64)
    out["mixed"] = v
    out["zeros"] = np.zeros(2049, np.uint64)
    out["huge"] = rng.integers(0, 2**62, 1500, dtype=np.uint64)
    out["one"] = np.array([7], np.uint64)
    out["bimodal"] = np.where(rng.random(3072) < 0.5, rng.integers(0, 4, 3072), rng.integers(1 << 15, 1 << 17, 3072)).astype(np.uint64)
    return out


# ------------------------------------------------------------------------- CPU ------------
def test_oracle_search_is_the_argmin_of_the_cost_table():
    v = streams()["mixed"]
    W, K, Cst = B.search(v)
    for b in range(len(W)):
        t = B.cost_table(v[b * 1024:(b + 1) * 1024])
        assert Cst[b] == t.min()
        assert t[W[b], K[b]] == t.min()
        # ties resolve to the smallest w, then the smallest k
        ws, ks = np.nonzero(t == t.min())
        assert (W[b], K[b]) == (ws[0], ks[0])


@pytest.mark.parametrize("name", ["geometric", "mixed", "zeros", "huge", "one", "bimodal"])
def test_oracle_block_stream_roundtrip(name):
    v = streams()[name]
    for W, K in (B.search(v)[:2], (np.zeros((v.size + 1023) // 1024, np.uint8), np.full((v.size + 1023) // 1024, 5, np.uint8)),
                 (np.full((v.size + 1023) // 1024, 32, np.uint8), np.full((v.size + 1023) // 1024, 31, np.uint8))):
        offs, pay, nbits = B.encode(v, W, K)
        assert nbits == sum(B.block_cost(v[b * 1024:(b + 1) * 1024], W[b], K[b]) for b in range(len(W)))
        assert np.array_equal(B.decode(pay, nbits, v.size, W, K, offs), v)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    f = B.features(streams()["mixed"])
    f = np.concatenate([f, rng.random((5, 34)).astype(np.float32)])
    p = B.init_params(2).astype(np.float64)
    p[B.OFF["b1"][0]:B.OFF["b1"][1]] = 0.05
    wl = rng.integers(0, 33, f.shape[0])
    kl = rng.integers(0, 32, f.shape[0])
    _, g = B.loss_and_grad(p, f, wl, kl, 1.0 / f.shape[0], exact=True)
    eps = 1e-6
    idx = list(rng.choice(np.flatnonzero(g), 40, replace=False))
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        num = (B.loss_and_grad(pp, f, wl, kl, 1.0 / f.shape[0], exact=True)[0] -
               B.loss_and_grad(pm, f, wl, kl, 1.0 / f.shape[0], exact=True)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(g[i]), (i, num, g[i])


def test_shipped_model_file_has_the_parameter_count():
    path = os.path.join(os.path.dirname(HERE), "xnyzip_b200", "model", "blockparams.f32")
    if not os.path.exists(path):
        pytest.skip("no trained model in the tree")
    assert os.path.getsize(path) == 4 * B.NPARAM


# ------------------------------------------------------------------------- GPU ------------
torch = None


def _t():
    global torch
    if torch is None:
        torch = pytest.importorskip("torch")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _dev(v):
    return _t().from_numpy(np.ascontiguousarray(v).view(np.int64)).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["geometric", "mixed", "zeros", "huge", "one", "bimodal"])
def test_search_cost_features_match_oracle(ctx, name):
    from xnyzip_b200 import _native as N
    T = _t()
    v = streams()[name]
    nb = (v.size + 1023) // 1024
    dv = _dev(v)
    w = T.zeros(nb, dtype=T.uint8, device="cuda")
    k = T.zeros(nb, dtype=T.uint8, device="cuda")
    c = T.zeros(nb, dtype=T.int32, device="cuda")
    f = T.zeros((nb, 34), dtype=T.float32, device="cuda")
    N.check(N.block_search(_ptr(dv), v.size, _ptr(w), _ptr(k), _ptr(c), None))
    N.check(N.block_features(_ptr(dv), v.size, _ptr(f), None))
    W, K, Cst = B.search(v)
    assert np.array_equal(w.cpu().numpy(), W) and np.array_equal(k.cpu().numpy(), K)
    assert np.array_equal(c.cpu().numpy(), Cst)
    np.testing.assert_allclose(f.cpu().numpy(), B.features(v), rtol=1e-5, atol=1e-6)
    # the cost of other pairs
    rng = np.random.default_rng(nb)
    W2 = rng.integers(0, 33, nb).astype(np.uint8)
    K2 = rng.integers(0, 32, nb).astype(np.uint8)
    dW2, dK2 = T.from_numpy(W2).cuda(), T.from_numpy(K2).cuda()  # kept alive until the kernel has run
    N.check(N.block_cost(_ptr(dv), v.size, _ptr(dW2), _ptr(dK2), _ptr(c), None))
    want = [B.block_cost(v[b * 1024:(b + 1) * 1024], W2[b], K2[b]) for b in range(nb)]
    assert c.cpu().numpy().tolist() == want


def _ext_stream(raw: bytes, direct: bool, rle: bool):
    """(meta, data) of the block-coded entry of an extended container."""
    import struct
    assert raw[:8] == b"XNYZBX01"
    p = 8 + 8
    (np_,) = struct.unpack_from("<Q", raw, p)
    p += 8 + 4 * np_ + 12 + 2
    if not direct:  # two bit-packed block streams first
        for _ in range(2):
            dl, ml = struct.unpack_from("<QQ", raw, p)
            p += 16 + ml + dl
    dl, ml = struct.unpack_from("<QQ", raw, p)
    p += 16
    return raw[p:p + ml], raw[p + ml:p + ml + dl]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 3])
@pytest.mark.parametrize("case", [("terrain", 1, 0.01, 1, 1), ("spheres", 1, 0.5, 0, 0), ("uniform", 0, 0.05, 0, 1),
                                  ("small", 1, 0.1, 1, 1)])
def test_extended_container_matches_oracle_and_decodes_like_the_reference(xnyz, ctx, oracle, mode, case):
    from xnyzip_b200 import synthetic as S
    T = _t()
    kind, q, l2, hil, rle = case
    x = {"terrain": lambda: S.terrain(120_000, 21, extent=3000.0, amplitude=20.0, wavelength=900.0),
         "spheres": lambda: S.spheres(90_000, 300, 22, extent=5000.0),
         "uniform": lambda: S.uniform(70_000, 23),
         "small": lambda: S.uniform(40_000, 24, 0.0, 60.0)}[kind]()
    ref_frame = ctx.compress(x, q, l2, hil, rle)
    ref_pts = ctx.decompress(ref_frame, q, l2, rle)
    ctx.set_block_mode(mode)
    try:
        raw = ctx.compress(x, q, l2, hil, rle, use_zstd=False)
        info = ctx.block_info()
        frame = ctx.compress(x, q, l2, hil, rle)
    finally:
        ctx.set_block_mode(0)
    assert info["mode"] == mode and info["values"] == ctx.last_info.num_units
    pts = ctx.decompress(frame, q, l2, rle)
    assert pts.tobytes() == ref_pts.tobytes()
    # the block-coded entry, byte for byte against the oracle's encoder of the same stream
    dx = T.from_numpy(x).cuda()
    buf = T.empty(x.shape[0], dtype=T.int64, device="cuda")  # no kernel: the library writes it on its stream
    cnt = ctx.stage_repos(dx.data_ptr(), x.shape[0], q, l2, hil, rle, buf.data_ptr(), x.shape[0])
    v = buf[:cnt].cpu().numpy().view(np.uint64)
    nb = (cnt + 1023) // 1024
    meta, data = _ext_stream(raw, ctx.last_info.is_direct == 1, rle == 1)
    w = np.frombuffer(data[:nb], np.uint8)
    k = np.frombuffer(data[nb:2 * nb], np.uint8)
    pad = (8 - (2 * nb) % 8) % 8
    offs = np.frombuffer(data[2 * nb + pad:2 * nb + pad + 8 * nb], np.uint64)
    if mode == 1:
        W, K, _ = B.search(v)
        assert np.array_equal(w, W) and np.array_equal(k, K)
    o_offs, o_pay, o_bits = B.encode(v, w, k)
    assert np.frombuffer(meta, np.uint64).tolist() == [cnt, o_bits]
    assert np.array_equal(offs, o_offs)
    assert data[2 * nb + pad + 8 * nb:] == o_pay


def _mlp_inputs(n, seed):
    rng = np.random.default_rng(seed)
    f = B.features(streams()["mixed"])
    f = np.concatenate([f, rng.random((n - f.shape[0], 34)).astype(np.float32)])
    p = B.init_params(seed)
    p[B.OFF["b1"][0]:B.OFF["b1"][1]] = rng.normal(0, 0.1, 64)
    p[B.OFF["b3"][0]:B.OFF["b3"][1]] = rng.normal(0, 0.1, 72)
    return f, p, rng.integers(0, 33, n).astype(np.uint8), rng.integers(0, 32, n).astype(np.uint8)


@pytest.mark.gpu
def test_mlp_forward_matches_oracle(ctx):
    from xnyzip_b200 import _native as N
    T = _t()
    n = 203
    f, p, _, _ = _mlp_inputs(n, 5)
    df, dp = T.from_numpy(f).cuda(), T.from_numpy(p).cuda()
    w = T.zeros(n, dtype=T.uint8, device="cuda")
    k = T.zeros(n, dtype=T.uint8, device="cuda")
    conf = T.zeros((n, 2), dtype=T.float32, device="cuda")
    lg = T.zeros((n, 65), dtype=T.float32, device="cuda")
    N.check(N.mlp_forward(_ptr(dp), _ptr(df), n, _ptr(w), _ptr(k), _ptr(conf), _ptr(lg), None))
    want, _ = B.forward(p, f)
    got = lg.cpu().numpy()
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 2e-2 * scale
    # argmax heads agree wherever the top two logits are not within the tolerance
    for lo, nn, out in ((0, 32, k), (32, 33, w)):
        z = want[:, lo:lo + nn]
        srt = np.sort(z, axis=1)
        clear = srt[:, -1] - srt[:, -2] > 4e-2 * scale
        assert np.array_equal(out.cpu().numpy()[clear], np.argmax(z, axis=1)[clear])
    c = conf.cpu().numpy()
    assert np.all((c > 0) & (c <= 1.0 + 1e-6))


@pytest.mark.gpu
def test_mlp_gradients_match_oracle(ctx):
    """Gradients of the tensor-core training kernel against the CPU oracle (same BF16
    roundings, float64 sums): relative L2 error per parameter tensor below 2%."""
    from xnyzip_b200 import _native as N
    T = _t()
    n = 237
    f, p, wl, kl = _mlp_inputs(n, 7)
    df, dp = T.from_numpy(f).cuda(), T.from_numpy(p).cuda()
    dw, dk = T.from_numpy(wl).cuda(), T.from_numpy(kl).cuda()
    grad = T.zeros_like(dp)
    loss = T.zeros(1, dtype=T.float32, device="cuda")
    gather = T.zeros(N.mlp_gather_floats(n), dtype=T.float32, device="cuda")
    N.check(N.mlp_train_batch(_ptr(dp), _ptr(df), _ptr(dw), _ptr(dk), None, 0, n, 1.0 / n, _ptr(grad), _ptr(loss),
                              _ptr(gather), None))
    wl_, g_ = B.loss_and_grad(p, f, wl, kl, 1.0 / n)
    got = grad.cpu().numpy().astype(np.float64)
    assert abs(float(loss.item()) - wl_) <= 1e-3 * abs(wl_)
    for name, (a, b) in B.OFF.items():
        err = np.linalg.norm(got[a:b] - g_[a:b]) / max(np.linalg.norm(g_[a:b]), 1e-12)
        assert err < 2e-2, (name, err)


@pytest.mark.gpu
def test_training_kernels_reduce_the_loss(ctx):
    """A few hundred Adam steps of the GPU kernels on labelled blocks lower the loss."""
    from xnyzip_b200 import _native as N
    from xnyzip_b200 import train_blockparams as TB
    T = _t()
    rng = np.random.default_rng(9)
    vals = np.concatenate([rng.geometric(pp, 1024).astype(np.uint64) for pp in rng.uniform(1e-4, 0.5, 300)])
    dv = _dev(vals)
    nb = vals.size // 1024
    F = T.zeros((nb, 34), dtype=T.float32, device="cuda")
    W = T.zeros(nb, dtype=T.uint8, device="cuda")
    K = T.zeros(nb, dtype=T.uint8, device="cuda")
    N.check(N.block_features(_ptr(dv), vals.size, _ptr(F), None))
    N.check(N.block_search(_ptr(dv), vals.size, _ptr(W), _ptr(K), None, None))
    prm, hist, _ = TB.train(F, W, K, epochs=40, batch=64, lr=3e-3, dev=T.device("cuda", 0), log=lambda *a: None)
    assert hist[-1] < 0.5 * hist[0], hist


@pytest.mark.gpu
def test_learned_mode_roundtrip_and_fallback(xnyz, ctx):
    from xnyzip_b200 import synthetic as S
    x = S.terrain(200_000, 31, extent=2000.0, amplitude=10.0, wavelength=700.0)
    ref = ctx.decompress(ctx.compress(x, 1, 0.01, 1, 1), 1, 0.01, 1)
    p = B.init_params(4)
    own = xnyz.Context(0)  # an untrained model on a context of its own
    try:
        for thr in (0.0, 1.0):  # no fallback / every block falls back to the exhaustive search
            own.set_model(p, thr)
            own.set_block_mode(2)
            fr = own.compress(x, 1, 0.01, 1, 1)
            info = own.block_info()
            assert ctx.decompress(fr, 1, 0.01, 1).tobytes() == ref.tobytes()
            assert info["fallback_blocks"] == (0 if thr == 0.0 else info["blocks"])
    finally:
        own.close()
