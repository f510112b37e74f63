"""The plain method at size against the reference: an 8M-point terrain cloud (the bench's
generator, seed 1) in all six variants of the bench (TO and cube x L2 {0.001, 0.01, 0.1},
Hilbert, -rle), through the device path and the host-buffer path, compared by SHA-256 with
what the reference itself produced on the same cloud (tests/golden/ref_digests.json, made by
tests/golden/make_ref_digests.py): the pre-zstd container, the zstd frame and the decoded
points, plus the L2 bound of every point (up to float32 resolution, xnyzip_b200.verify)."""
import json
import os

import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(__file__))
KEY = "terrain_8000000_seed1"
VARIANTS = [(1, 0.001), (1, 0.01), (1, 0.1), (0, 0.001), (0, 0.01), (0, 0.1)]


@pytest.fixture(scope="module")
def cloud():
    from xnyzip_b200 import synthetic as S
    from xnyzip_b200 import verify as V
    with open(os.path.join(HERE, "golden", "ref_digests.json")) as f:
        ref = json.load(f)[KEY]
    x = S.terrain(ref["points"], ref["seed"])
    assert V.sha256(x) == ref["input_sha256"], "the generator did not reproduce the reference's input cloud"
    return x, ref


@pytest.mark.parametrize("q,l2", VARIANTS)
def test_terrain_8m_matches_reference(ctx, cloud, q, l2):
    from xnyzip_b200 import verify as V
    x, ref = cloud
    want = ref["variants"][f"{'to' if q else 'cube'}_{l2}"]
    n = x.shape[0]
    d = torch.from_numpy(x).cuda()
    p, ln = ctx.compress_device(d.data_ptr(), n, q, l2, True, True)
    torch.cuda.synchronize()
    assert ln == want["container_bytes"]
    assert V.sha256(V.device_view(p, (ln,), "|u1", d.device)) == want["container_sha256"]
    dp, nout = ctx.decompress_device(p, ln, q, l2, True)
    torch.cuda.synchronize()
    dec = V.device_view(dp, (nout, 3), "<f4", d.device).clone()
    assert nout == want["points_out"]
    assert V.sha256(dec) == want["points_sha256"]
    # the host-buffer path: host points in, the zstd frame out, host points back
    frame = ctx.compress(x, q, l2, True, True)
    assert len(frame) == want["frame_bytes"] and V.sha256(frame) == want["frame_sha256"]
    back = ctx.decompress(frame, q, l2, True)
    assert V.sha256(back) == want["points_sha256"]
    # every point within its bound up to the float32 resolution of the reference's arithmetic
    # on a 10 km cloud (a 1 mm bound is below it: the reference's own decoded points, which
    # these are, exceed 1 mm for many points)
    rep = V.l2_report(ctx, d, q, l2, decoded=dec)
    assert rep["over_bound_plus_slack"] == 0, rep
    assert rep["mismatch"] == rep["z_minus1_points"], rep
