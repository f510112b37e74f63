"""Seeded synthetic point clouds standing in for the reference's datasets.

The reference measures on USGS LiDAR and a vesicle surface set that are not available
here; these generators reproduce their shapes, sizes and value distributions:

  * uniform(n, seed)       - i.i.d. uniform in [0, 1000]^3 (the small plain-method case)
  * terrain(n, seed)       - LiDAR-like terrain: x,y uniform over [0, 10000]^2 m, z a sum of
                             8 random sinusoid octaves (amplitude 50 m halving per octave,
                             wavelength 5000 m halving, random phase and direction) plus
                             N(0, 0.1^2) noise; 5% of the points are copies of base points
                             with z lowered by U(0, 2) m (multi-return), appended last
  * spheres(n, k, seed)    - points on k sphere surfaces: centres uniform in [0, 1e5]^3,
                             radii lognormal(ln 20, 0.4), points per sphere proportional to
                             r^2 (largest remainder), radial jitter N(0, 0.2^2)
All return float32 arrays of shape (n, 3).
"""
from __future__ import annotations

import numpy as np


def uniform(n: int, seed: int = 0, lo: float = 0.0, hi: float = 1000.0) -> np.ndarray:
    return np.random.default_rng(seed).uniform(lo, hi, (n, 3)).astype(np.float32)


def terrain(n: int, seed: int = 1, extent: float = 10000.0, amplitude: float = 50.0, wavelength: float = 5000.0,
            dup_fraction: float = 0.05, chunk: int = 1 << 22) -> np.ndarray:
    rng = np.random.default_rng(seed)
    ndup = int(round(n * dup_fraction))
    nbase = n - ndup
    ang = rng.uniform(0.0, 2.0 * np.pi, 8)
    dirs = np.stack([np.cos(ang), np.sin(ang)], axis=1)
    phase = rng.uniform(0.0, 2.0 * np.pi, 8)
    amp = amplitude * 0.5 ** np.arange(8)
    lam = wavelength * 0.5 ** np.arange(8)
    out = np.empty((n, 3), dtype=np.float32)
    xy = rng.uniform(0.0, extent, (nbase, 2))
    noise = rng.normal(0.0, 0.1, nbase)
    for s in range(0, nbase, chunk):
        e = min(nbase, s + chunk)
        p = xy[s:e]
        z = noise[s:e].copy()
        for k in range(8):
            z += amp[k] * np.sin(2.0 * np.pi * (p @ dirs[k]) / lam[k] + phase[k])
        out[s:e, 0:2] = p
        out[s:e, 2] = z
    if ndup:
        src = rng.integers(0, nbase, ndup)
        out[nbase:] = out[src]
        out[nbase:, 2] = (out[src, 2].astype(np.float64) - rng.uniform(0.0, 2.0, ndup)).astype(np.float32)
    return out


def spheres(n: int, k: int = 200_000, seed: int = 2, extent: float = 1e5, r_median: float = 20.0,
            r_sigma: float = 0.4, jitter: float = 0.2) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, extent, (k, 3))
    radii = rng.lognormal(np.log(r_median), r_sigma, k)
    w = radii ** 2
    quota = w / w.sum() * n
    counts = np.floor(quota).astype(np.int64)
    rest = n - int(counts.sum())
    if rest:
        counts[np.argsort(-(quota - counts), kind="stable")[:rest]] += 1
    owner = np.repeat(np.arange(k), counts)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = radii[owner] + rng.normal(0.0, jitter, n)
    return (centres[owner] + r[:, None] * u).astype(np.float32)


def planar(n: int, seed: int = 3, extent: float = 200.0, z: float = 5.0) -> np.ndarray:
    """All points at one height: many land exactly on the lowest z plane after shifting."""
    x = np.random.default_rng(seed).uniform(0.0, extent, (n, 3)).astype(np.float32)
    x[:, 2] = z
    return x


def with_duplicates(n: int, seed: int = 4, extent: float = 50.0, max_repeat: int = 40) -> np.ndarray:
    """Few distinct points repeated many times (long -rle runs)."""
    rng = np.random.default_rng(seed)
    base = rng.uniform(0.0, extent, (max(1, n // 8), 3)).astype(np.float32)
    reps = rng.integers(1, max_repeat, base.shape[0])
    x = np.repeat(base, reps, axis=0)
    return x[:n] if x.shape[0] >= n else np.concatenate([x, base[: n - x.shape[0]]])
