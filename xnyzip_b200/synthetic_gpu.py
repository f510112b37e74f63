"""Seeded synthetic point clouds drawn on the GPU with torch (fast generation of many and
large clouds for training data and the batched workload).

The shapes follow xnyzip_b200.synthetic (the same distributions, not the same numbers):
  * gen_uniform(n, seed)  - i.i.d. uniform in [0, 1000]^3
  * gen_terrain(n, seed)  - terrain: x,y uniform over [0, extent]^2, z = 8 sinusoid octaves
                            (amplitude halving, wavelength halving, random phase/direction)
                            + N(0, 0.1^2); a fraction of multi-return copies with z - U(0, 2)
  * gen_spheres(n, seed)  - points on k sphere surfaces (lognormal radii, counts ~ r^2)
  * batch_clouds(count)   - the uneven batch: point counts log-uniform in [1e3, 4e6], terrain or
                            clustered with p = 0.5, bbox side log-uniform in [10, 1e4] (terrain
                            amplitudes scaled by side / 1e4; clustered with max(1, n / 875)
                            spheres, radii scaled by side / 1e5), L2 bound from {0.001, 0.01,
                            0.1}; cloud c uses seed 1000 + c
"""
from __future__ import annotations

import math

import numpy as np


def _torch():
    import torch
    return torch


def gen_uniform(n, seed, dev):
    torch = _torch()
    g = torch.Generator(device=dev).manual_seed(seed)
    return torch.rand((n, 3), generator=g, device=dev, dtype=torch.float64).mul_(1000.0).float()


def gen_terrain(n, seed, dev, extent=10000.0, amplitude=50.0, wavelength=5000.0, dup=0.05):
    torch = _torch()
    g = torch.Generator(device=dev).manual_seed(seed)
    nd = int(round(n * dup))
    nb = n - nd
    ang = torch.rand(8, generator=g, device=dev, dtype=torch.float64) * 2 * math.pi
    ph = torch.rand(8, generator=g, device=dev, dtype=torch.float64) * 2 * math.pi
    xy = torch.rand((nb, 2), generator=g, device=dev, dtype=torch.float64) * extent
    z = torch.randn(nb, generator=g, device=dev, dtype=torch.float64) * 0.1
    for k in range(8):
        d = torch.stack([torch.cos(ang[k]), torch.sin(ang[k])])
        z += amplitude * 0.5 ** k * torch.sin(2 * math.pi * (xy @ d) / (wavelength * 0.5 ** k) + ph[k])
    base = torch.cat([xy, z[:, None]], 1).float()
    if nd:
        src = torch.randint(0, nb, (nd,), generator=g, device=dev)
        cp = base[src].clone()
        cp[:, 2] = (cp[:, 2].double() - torch.rand(nd, generator=g, device=dev, dtype=torch.float64) * 2).float()
        base = torch.cat([base, cp], 0)
    return base.contiguous()


def gen_spheres(n, seed, dev, k=20000, extent=1e5, r_median=20.0, r_sigma=0.4, jitter=0.2):
    torch = _torch()
    g = torch.Generator(device=dev).manual_seed(seed)
    c = torch.rand((k, 3), generator=g, device=dev, dtype=torch.float64) * extent
    r = torch.exp(math.log(r_median) + r_sigma * torch.randn(k, generator=g, device=dev, dtype=torch.float64))
    w = r * r
    quota = w / w.sum() * n
    cnt = torch.floor(quota).long()
    rest = n - int(cnt.sum())
    if rest:
        cnt[torch.argsort(-(quota - cnt), stable=True)[:rest]] += 1
    owner = torch.repeat_interleave(torch.arange(k, device=dev), cnt)
    u = torch.randn((n, 3), generator=g, device=dev, dtype=torch.float64)
    u /= u.norm(dim=1, keepdim=True)
    rr = r[owner] + jitter * torch.randn(n, generator=g, device=dev, dtype=torch.float64)
    return (c[owner] + rr[:, None] * u).float().contiguous()


def block_key_bits(extent, l2: float) -> int:
    """Sort-key bits of block mode (truncated octahedron) for a bounding box of the given
    side lengths: bit length of the 128^3 super-block count, plus 21."""
    div = 2.0 * l2 / math.sqrt(5.0)
    cells = [extent[0] / (2 * div), extent[1] / (2 * div), extent[2] / div]
    nb = 1
    for c in cells:
        nb *= int(c) // 128 + 1
    return max(1, (nb - 1).bit_length()) + 21


def batch_clouds(count: int, dev, seed0: int = 1000, lo: float = 1e3, hi: float = 4e6):
    """[(points tensor (n, 3) float32 on dev, l2)] of the uneven batch.  A cloud whose block
    sort keys would need more than 63 bits at its drawn bound (a clustered cloud with a
    bounding box above ~3.5 km at L2 0.001) takes the next coarser bound instead."""
    out = []
    for c in range(count):
        rng = np.random.default_rng(seed0 + c)
        n = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        side = math.exp(rng.uniform(math.log(10.0), math.log(1e4)))
        l2 = float(rng.choice([0.001, 0.01, 0.1]))
        s = int(rng.integers(0, 2**31 - 1))
        if rng.random() < 0.5:
            pts = gen_terrain(n, s, dev, extent=side, amplitude=50.0 * side / 1e4, wavelength=5000.0 * side / 1e4)
        else:
            pts = gen_spheres(n, s, dev, k=max(1, n // 875), extent=side, r_median=20.0 * side / 1e5)
        ext = (pts.max(0).values - pts.min(0).values).double().cpu().tolist()
        while l2 < 0.1 and block_key_bits(ext, l2) > 63:
            l2 *= 10.0
        out.append((pts, l2))
    return out
