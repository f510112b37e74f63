"""The oracle restatement against the reference's own outputs (CPU).

Pins: (1) the committed fixtures generated by the reference itself
(tests/golden/make_golden.py) and (2), where the reference is built here (oracle/_ref),
a direct byte comparison on a matrix of inputs and modes.
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import quiet_call, small_inputs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_fixtures.npz")
Q = {0: "cube", 1: "to", 2: "adaptive"}


def golden_cases():
    f = np.load(GOLDEN)
    for name in f["names"]:
        name = str(name)
        q, hil, rle, th = (int(v) for v in f[f"{name}/params"])
        yield name, f[f"{name}/points"], Q[q], float(f[f"{name}/l2"][0]), hil, rle, th, f


@pytest.mark.parametrize("case", [c[0] for c in golden_cases()])
def test_oracle_matches_reference_fixture(oracle, case):
    for name, x, q, l2, hil, rle, th, f in golden_cases():
        if name != case:
            continue
        frame = oracle.compress(x, q, l2, hil, rle, th, zstd=True)
        assert frame == f[f"{name}/frame"].tobytes()
        raw = oracle.compress(x, q, l2, hil, rle, th, zstd=False)
        assert raw == f[f"{name}/container"].tobytes()
        dec = oracle.decompress(frame, q, l2, rle)
        assert dec.tobytes() == f[f"{name}/decoded"].tobytes()


def test_oracle_config1_digest(oracle):
    from xnyzip_b200 import synthetic as S
    f = np.load(GOLDEN)
    x = S.uniform(1_000_000, 0)
    assert hashlib.sha256(x.tobytes()).digest() == f["config1/input_sha256"].tobytes()
    frame = oracle.compress(x, "to", 0.05, 0, 1, 1024)
    assert len(frame) == int(f["config1/frame_len"][0])
    assert hashlib.sha256(frame).digest() == f["config1/frame_sha256"].tobytes()
    dec = oracle.decompress(frame, "to", 0.05, 1)
    assert hashlib.sha256(dec.tobytes()).digest() == f["config1/decoded_sha256"].tobytes()


MODES = [(q, l2, hil, rle, th) for q in ("to", "cube", "adaptive") for l2 in (0.05, 0.5) for hil in (0, 1) for rle in (0, 1)
         for th in (1024, 0)]


@pytest.mark.parametrize("kind", list(small_inputs(16).keys()))
def test_oracle_vs_reference_matrix(oracle, reference, kind):
    x = small_inputs(3000)[kind]
    for q, l2, hil, rle, th in MODES:
        a = quiet_call(reference, reference.compress, x, q, l2, hil, rle, th)
        b = oracle.compress(x, q, l2, hil, rle, th)
        assert a == b, (kind, q, l2, hil, rle, th)
        da = quiet_call(reference, reference.decompress, a, q, l2, rle)
        db = oracle.decompress(b, q, l2, rle)
        assert da.tobytes() == db.tobytes(), (kind, q, l2, hil, rle, th)


def test_oracle_hilbert_vs_reference(oracle, reference):
    codes = np.arange(1 << 18, dtype=np.uint64)
    assert np.array_equal(oracle.m2h(codes, 20), reference.m2h(codes, 20))
    assert np.array_equal(oracle.h2m(codes, 20), reference.h2m(codes, 20))
    rng = np.random.default_rng(9)
    for it in range(1, 21):
        c = rng.integers(0, 2**63, 4000, dtype=np.uint64)
        assert np.array_equal(oracle.m2h(c, it), reference.m2h(c, it))
        assert np.array_equal(oracle.h2m(c, it), reference.h2m(c, it))


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_oracle_huffman_vs_reference(oracle, reference, kind):
    rng = np.random.default_rng(kind)
    data = {
        0: [rng.integers(0, 256, 5000), rng.geometric(0.3, 5000) % 256, np.zeros(100), np.array([7])],
        1: [rng.integers(1, 9, 5000), np.full(50, 3), rng.integers(1, 3, 77)],
        2: [rng.geometric(0.5, 5000), rng.integers(1, 5000, 3000), np.ones(10)],
    }[kind]
    for d in data:
        for eg in (False, True):
            a = quiet_call(reference, reference.huffman, d, kind, eg)
            b = oracle.huffman(d, kind, eg)
            assert a == b


def test_oracle_gr_and_bitpack_vs_reference(oracle, reference):
    rng = np.random.default_rng(3)
    for d in (rng.integers(255, 1 << 18, 3000), rng.integers(0, 5, 100), np.array([], np.uint64),
              np.array([2**40, 300, 301], np.uint64)):
        assert oracle.gr_pack(d) == reference.gr_pack(d)
        if d.size:
            assert oracle.bitpack(d) == reference.bitpack(d)


def test_oracle_shared_codebook_fixture(oracle):
    """fit_profile / compress_with_profile (composer/block_compressor.hpp:241-431): the
    restatement reproduces the reference's frames and profile bytes."""
    f = np.load(GOLDEN)
    frame, prof = oracle.fit_profile(f["profile/fit_points"], "to", 0.05, 1)
    assert frame == f["profile/fit_frame"].tobytes()
    assert prof == f["profile/profile"].tobytes()
    for i in range(2):
        got = oracle.compress_with_profile(f[f"profile/points{i}"], "to", 0.05, 1, prof)
        assert got == f[f"profile/frame{i}"].tobytes()


def test_oracle_shared_codebook_vs_reference(oracle, reference):
    from xnyzip_b200 import synthetic as S
    fit_x = S.terrain(6000, 51, extent=300.0, amplitude=3.0, wavelength=150.0)
    others = [S.uniform(4000, 52), S.spheres(5000, 12, 53, extent=150.0)]
    for q in ("to", "cube", "adaptive"):
        for hil in (0, 1):
            a = oracle.fit_profile(fit_x, q, 0.1, hil)
            b = quiet_call(reference, reference.fit_profile, fit_x, q, 0.1, hil)
            assert a == b, (q, hil)
            for x in others:
                assert oracle.compress_with_profile(x, q, 0.1, hil, b[1]) == \
                    quiet_call(reference, reference.compress_with_profile, x, q, 0.1, hil, b[1]), (q, hil)
