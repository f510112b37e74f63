"""Distributed-RLE cell tables through the C ABI against the reference built from its own
sources (composer/block_compressor_rle.hpp:341-470 encode_cells_with_counts,
composer/block_decompressor_rle.hpp:230-358 decompress_to_cells / expand_cells_to_points):
byte-identical frames, identical cell tables, bit-identical expanded points."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tables(reference):
    from conftest import quiet_call
    from xnyzip_b200 import synthetic as S
    out = []
    for name, x, q, l2 in [("terrain", S.terrain(60_000, 5, extent=400.0, amplitude=4.0, wavelength=150.0), "to", 0.05),
                           ("spheres", S.spheres(40_000, 30, 6, extent=2000.0), "to", 0.5),
                           ("dups", S.with_duplicates(30_000, 7), "cube", 0.05),
                           ("planar", S.planar(20_000, 8), "to", 0.05)]:
        off, qc = quiet_call(reference, reference.quantize, x, q, l2)
        cells, counts = np.unique(qc, axis=0, return_counts=True)
        rng = np.maximum(qc.max(axis=0), 0)
        # a few large counts (the count stream's sparse table / exp-Golomb switch)
        counts = counts.astype(np.int32)
        counts[::97] += np.arange(counts[::97].size, dtype=np.int32) * 1009
        out.append((name, cells.astype(np.int32), counts, rng.astype(np.int32), off, q, l2))
    return out


@pytest.mark.parametrize("hilbert", [0, 1])
def test_cells_roundtrip_matches_reference(ctx, reference, hilbert):
    from conftest import quiet_call
    for name, cells, counts, rng, off, q, l2 in _tables(reference):
        perm = np.random.default_rng(len(cells)).permutation(len(cells))  # input order is free
        cells, counts = cells[perm], counts[perm]
        want = quiet_call(reference, reference.encode_cells, cells, counts, rng, off, hilbert)
        got = ctx.encode_cells(cells, counts, rng, off, hilbert)
        assert got == want, name
        c2, k2, o2, r2, h2 = ctx.decompress_to_cells(got)
        rc, rk, ro, rr, rh = quiet_call(reference, reference.decompress_to_cells, want)
        assert np.array_equal(c2, rc) and np.array_equal(k2, rk), name
        assert o2.tobytes() == ro.tobytes() and np.array_equal(r2, rr) and h2 == rh
        pts = ctx.expand_cells(c2, k2, o2, {"cube": 0, "to": 1}[q], l2)
        assert pts.tobytes() == quiet_call(reference, reference.expand_cells, rc, rk, ro, q, l2).tobytes(), name
        # expand_cells_to_points has no adaptive branch: the cube quantizer recovers the cells
        pts = ctx.expand_cells(c2, k2, o2, 2, l2)
        assert pts.tobytes() == quiet_call(reference, reference.expand_cells, rc, rk, ro, "adaptive", l2).tobytes()


def test_cells_reject_direct_and_out_of_range(ctx, xnyz):
    x = np.random.default_rng(2).uniform(0, 5, (5000, 3)).astype(np.float32)
    direct_frame = ctx.compress(x, 1, 0.05, 0, 1)  # small extent: direct mode
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.decompress_to_cells(direct_frame)
    assert e.value.status == 2
    cells = np.array([[0, 0, 0], [5, 1, 1]], np.int32)
    with pytest.raises(xnyz.XnyzError) as e:
        ctx.encode_cells(cells, np.ones(2, np.int32), np.array([3, 3, 3], np.int32), np.zeros(3, np.float32), 0)
    assert e.value.status == 6
