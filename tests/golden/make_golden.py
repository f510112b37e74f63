"""Generates tests/golden/reference_fixtures.npz from the reference itself.

The reference (compiled from its own sources into oracle/_ref by oracle/build_ref.sh)
compresses a set of small seeded inputs; the fixture keeps each input, the reference's
zstd frame, its pre-zstd container and the points its decompressor returns.  Tests check the
oracle restatement and the GPU path against these bytes on machines without the reference.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from oracle import Reference  # noqa: E402
from xnyzip_b200 import synthetic as S  # noqa: E402

# (name, points, quantizer, l2, hilbert, rle, direct_threshold)
def cases():
    rng = np.random.default_rng(11)
    yield "uniform_to_z_rle", S.uniform(1500, 21), "to", 0.05, 0, 1, 1024
    yield "uniform_cube_h_normal", S.uniform(1500, 22), "cube", 0.05, 1, 0, 1024
    yield "terrain_to_h_rle", S.terrain(1500, 23, extent=300.0, amplitude=3.0, wavelength=150.0), "to", 0.01, 1, 1, 1024
    yield "terrain_cube_h_rle", S.terrain(1500, 24, extent=300.0, amplitude=3.0, wavelength=150.0), "cube", 0.1, 1, 1, 1024
    yield "spheres_to_z_normal", S.spheres(1500, 10, 25, extent=300.0), "to", 0.5, 0, 0, 1024
    yield "direct_to_h_rle", rng.uniform(0, 3, (1500, 3)).astype(np.float32), "to", 0.05, 1, 1, 1024
    yield "direct_cube_z_normal", rng.uniform(0, 3, (1500, 3)).astype(np.float32), "cube", 0.05, 0, 0, 1024
    yield "planar_to_z_rle", S.planar(1500, 26), "to", 0.05, 0, 1, 1024
    yield "planar_to_h_normal_direct", S.planar(1500, 27, extent=20.0), "to", 0.05, 1, 0, 1024
    yield "duplicates_to_h_rle", S.with_duplicates(1500, 28), "to", 0.05, 1, 1, 1024
    base = rng.uniform(0, 100, (150, 3)).astype(np.float32)
    yield "egcounts_to_h_rle", np.repeat(base, rng.integers(1, 90, 150), axis=0), "to", 0.01, 1, 1, 1024
    yield "single_point", np.array([[1.5, -2.0, 3.25]], np.float32), "to", 0.05, 0, 1, 1024
    # AdaptiveQuantizer (quantizer/adaptive_quantizer.hpp): steps in the params, block and
    # direct mode, a flat axis (extent = the smallest normal float), and -rle, whose decoder
    # recovers the cells with the cube quantizer (block_decompressor_rle.hpp:189-196)
    yield "terrain_adaptive_h_normal", S.terrain(1500, 29, extent=300.0, amplitude=3.0, wavelength=150.0), \
        "adaptive", 0.05, 1, 0, 1024
    yield "direct_adaptive_z_normal", rng.uniform(0, 3, (1500, 3)).astype(np.float32), "adaptive", 0.05, 0, 0, 1024
    flat = rng.uniform(0, 200, (1500, 3)).astype(np.float32)
    flat[:, 2] = 4.25
    yield "flat_adaptive_h_normal", flat, "adaptive", 0.01, 1, 0, 1024
    yield "uniform_adaptive_h_rle", S.uniform(1500, 30), "adaptive", 0.05, 1, 1, 1024


def main():
    ref = Reference()
    out = {}
    names = []
    for name, x, q, l2, hil, rle, th in cases():
        ref.quiet(True)
        try:
            frame = ref.compress(x, q, l2, hil, rle, th)
            raw = ref.unzstd(frame)
            dec = ref.decompress(frame, q, l2, rle)
        finally:
            ref.quiet(False)
        names.append(name)
        out[f"{name}/points"] = x
        out[f"{name}/params"] = np.array([{"cube": 0, "to": 1, "adaptive": 2}[q], hil, rle, th], np.int64)
        out[f"{name}/l2"] = np.array([l2], np.float32)
        out[f"{name}/frame"] = np.frombuffer(frame, np.uint8)
        out[f"{name}/container"] = np.frombuffer(raw, np.uint8)
        out[f"{name}/decoded"] = dec
        print(f"{name}: {x.shape[0]} points -> {len(frame)} B frame, {len(raw)} B container, "
              f"sha256 {hashlib.sha256(frame).hexdigest()[:12]}")
    # config 1 of the plain method at full size: only digests (the frame is 3.4 MB)
    x = S.uniform(1_000_000, 0)
    ref.quiet(True)
    try:
        frame = ref.compress(x, "to", 0.05, 0, 1, 1024)
        dec = ref.decompress(frame, "to", 0.05, 1)
    finally:
        ref.quiet(False)
    out["config1/frame_sha256"] = np.frombuffer(hashlib.sha256(frame).digest(), np.uint8)
    out["config1/frame_len"] = np.array([len(frame)], np.int64)
    out["config1/decoded_sha256"] = np.frombuffer(hashlib.sha256(dec.tobytes()).digest(), np.uint8)
    out["config1/input_sha256"] = np.frombuffer(hashlib.sha256(x.tobytes()).digest(), np.uint8)
    # shared codebooks (block_compressor.hpp:241-431): a profile fit on one terrain chunk,
    # then two other chunks (one with a range below the direct threshold) coded with it
    fit_x = S.terrain(3000, 31, extent=300.0, amplitude=3.0, wavelength=150.0)
    others = [S.terrain(2500, 32, extent=300.0, amplitude=3.0, wavelength=150.0),
              np.random.default_rng(33).uniform(0, 3, (1200, 3)).astype(np.float32)]
    ref.quiet(True)
    try:
        fit_frame, prof = ref.fit_profile(fit_x, "to", 0.05, 1)
        with_frames = [ref.compress_with_profile(x, "to", 0.05, 1, prof) for x in others]
    finally:
        ref.quiet(False)
    out["profile/fit_points"] = fit_x
    out["profile/fit_frame"] = np.frombuffer(fit_frame, np.uint8)
    out["profile/profile"] = np.frombuffer(prof, np.uint8)
    for i, (x, fr) in enumerate(zip(others, with_frames)):
        out[f"profile/points{i}"] = x
        out[f"profile/frame{i}"] = np.frombuffer(fr, np.uint8)
    print(f"profile: {len(prof)} B profile, frames {len(fit_frame)} / {[len(f) for f in with_frames]} B")
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "reference_fixtures.npz"), **out)
    print("config1:", len(frame), "B frame")


if __name__ == "__main__":
    main()
