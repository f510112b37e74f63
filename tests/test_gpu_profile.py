"""Shared codebooks on the GPU path (BlockCompressor::fit_profile / compress_with_profile,
composer/block_compressor.hpp:241-431): frames and profile bytes identical to the reference's
fixtures and to the reference built here, decoded points identical, the rejected cases."""
import numpy as np
import pytest

from conftest import quiet_call

pytestmark = pytest.mark.gpu

GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden", "reference_fixtures.npz")


def test_gpu_profile_matches_fixture(ctx):
    f = np.load(GOLDEN)
    frame, prof = ctx.fit_profile(f["profile/fit_points"], 1, 0.05, 1)
    assert frame == f["profile/fit_frame"].tobytes()
    assert prof == f["profile/profile"].tobytes()
    for i in range(2):
        got = ctx.compress_with_profile(f[f"profile/points{i}"], 1, 0.05, 1, prof)
        assert got == f[f"profile/frame{i}"].tobytes()
        dec = ctx.decompress(got, 1, 0.05, 0)
        assert dec.shape == f[f"profile/points{i}"].shape


@pytest.mark.parametrize("q", [0, 1, 2])
def test_gpu_profile_matches_reference(ctx, reference, q):
    from xnyzip_b200 import synthetic as S
    qn = {0: "cube", 1: "to", 2: "adaptive"}[q]
    fit_x = S.terrain(40_000, 61, extent=500.0, amplitude=5.0, wavelength=250.0)
    others = [S.terrain(30_000, 62, extent=500.0, amplitude=5.0, wavelength=250.0), S.uniform(20_000, 63),
              np.random.default_rng(64).uniform(0, 4, (5000, 3)).astype(np.float32)]
    for hil in (0, 1):
        frame, prof = ctx.fit_profile(fit_x, q, 0.02, hil)
        rframe, rprof = quiet_call(reference, reference.fit_profile, fit_x, qn, 0.02, hil)
        assert prof == rprof and frame == rframe, (qn, hil)
        for x in others:
            got = ctx.compress_with_profile(x, q, 0.02, hil, prof)
            want = quiet_call(reference, reference.compress_with_profile, x, qn, 0.02, hil, prof)
            assert got == want, (qn, hil, x.shape)
            dg = ctx.decompress(got, q, 0.02, 0)
            dr = quiet_call(reference, reference.decompress, want, qn, 0.02, 0)
            assert dg.tobytes() == dr.tobytes()


def test_gpu_profile_reorders_like_compress(ctx):
    import xnyzip_b200 as X
    from xnyzip_b200 import synthetic as S
    x = S.terrain(10_000, 65, extent=300.0, amplitude=3.0, wavelength=150.0)
    a, b = x.copy(), x.copy()
    bc = X.BlockCompressor(X.QUANTIZER_TYPE.TRUNCATED_OCTAHEDRON, 0.05, context=ctx)
    frame, prof = bc.fit_profile(a, True)
    frame2 = bc.compress_with_profile(b, True, prof)
    # the loaded table is written back in its own iteration order, so the bytes differ, but
    # both frames hold the same codes and decode to the same points
    d1 = ctx.decompress(frame, 1, 0.05, 0)
    d2 = ctx.decompress(frame2, 1, 0.05, 0)
    assert d1.tobytes() == d2.tobytes()
    assert np.array_equal(a, b) and not np.array_equal(a, x)


def test_gpu_profile_rejects(ctx, xnyz):
    from xnyzip_b200 import synthetic as S
    x = S.uniform(2000, 66)
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.compress_with_profile(x, 1, 0.05, 1, b"")
    assert e.value.status == 1
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.compress_with_profile(x, 1, 0.05, 1, b"\x05\x00\x00\x00ab")
    assert e.value.status == 1
    # a profile whose repos codebook lacks a symbol of the chunk
    _, prof = ctx.fit_profile(x, 1, 0.05, 1)
    n0 = int.from_bytes(prof[:4], "little")
    small = (4).to_bytes(4, "little") + b"\x00\x00\x00\x00" + prof[4 + n0:]
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.compress_with_profile(x, 1, 0.05, 1, small)
    assert e.value.status == 1
