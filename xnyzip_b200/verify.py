"""Checks of a decoded cloud against its input, on the device.

The reference reports, for a -normal round trip, the L2 error of every point against its
decoded counterpart, the count above the bound and the maximum (main.cpp:162-198, in float:
``(p - r).norm()``, Eigen's norm being ``sqrt(c0 + (c1 + c2))``); for -rle it reports
nothing, since the decoded cloud lists unique cells and no longer lines up with the input.
These checks work for both container kinds:

* every input point p_i is quantized and recovered by the library's own stage kernels
  (xnyz_stage_quantize / xnyz_stage_recover), r_i = recover(quantize(p_i)), and the float
  error |p_i - r_i| is taken the way main.cpp takes it;
* the decoded cloud must be the multiset {r_i} (a -normal container reorders the points,
  a -rle container repeats each cell's point by its count), compared through a 64-bit hash
  of each point's bits;
* float32 resolution: the reference quantizes and recovers in float32, so on a cloud whose
  extent E is large against the bound the lattice index p / step is itself rounded (its
  spacing is ulp(E / step) steps) and so are the shift (ulp(E)) and the unshift (ulp(M), M the
  largest coordinate).  The report gives that slack, sqrt(3) * (step * ulp(E / step) + ulp(E)
  + ulp(M)), and counts the points beyond
  bound + slack, which must be none; points between the bound and bound + slack are the
  reference's own (its decoded points are these, bit for bit);
* points whose truncated-octahedron cell has z = -1 (a point on the bottom face of the
  bounding box, where round(-0.5) = -1) are counted apart: the reference's block arithmetic
  wraps their block id and decodes them far away, and this path reproduces that.

Used by bench.py and the tests; everything runs in torch on the device that holds the
points, on the caller's current stream.
"""
from __future__ import annotations

import ctypes as C
import hashlib

import numpy as np

from . import _native as N

_MASK32 = 0xFFFFFFFF


def _s64(c: int) -> int:
    return c - (1 << 64) if c >= (1 << 63) else c


_K = [_s64(c) for c in (0x9E3779B97F4A7C15, 0xC2B2AE3D27D4EB4F, 0x165667B19E3779F9, 0xBF58476D1CE4E5B9,
                        0x94D049BB133111EB)]


class _DeviceArray:
    """A raw device pointer as a __cuda_array_interface__ object (no copy)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"data": (int(ptr), False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 3, "strides": None}


def device_view(ptr: int, shape, dtype: str, device):
    """A torch tensor over library-owned device memory (valid until the next call on the
    context that owns it).  dtype: '<f4', '|u1', ..."""
    import torch
    if int(np.prod(shape)) == 0:
        return torch.empty(shape, dtype={"<f4": torch.float32, "|u1": torch.uint8}[dtype], device=device)
    return torch.as_tensor(_DeviceArray(ptr, shape, dtype), device=device)


def sha256(t) -> str:
    """SHA-256 of a tensor's (or array's / bytes') raw bytes."""
    if isinstance(t, (bytes, bytearray, memoryview)):
        return hashlib.sha256(t).hexdigest()
    if not isinstance(t, np.ndarray):
        t = t.contiguous().cpu().numpy()
    return hashlib.sha256(memoryview(np.ascontiguousarray(t)).cast("B")).hexdigest()


def _row_hash(pts):
    """64-bit mix of each point's three float bit patterns (int64, wrapping arithmetic)."""
    import torch
    b = pts.contiguous().view(torch.int32).to(torch.int64) & _MASK32
    h = b[:, 0] * _K[0] + b[:, 1] * _K[1] + b[:, 2] * _K[2]
    h = h ^ ((h >> 31) & ((1 << 33) - 1))
    h = h * _K[3]
    h = h ^ ((h >> 29) & ((1 << 35) - 1))
    h = h * _K[4]
    return h ^ ((h >> 32) & _MASK32)


def multiset_mismatch(a, b) -> int:
    """Points of `a` not matched one to one by an equal point of `b` (bit patterns), through
    a 64-bit hash of each point: 0 when the two clouds are the same multiset."""
    import torch
    ha, hb = torch.sort(_row_hash(a)).values, torch.sort(_row_hash(b)).values
    if ha.shape == hb.shape and bool(torch.equal(ha, hb)):
        return 0
    u = torch.unique(torch.cat([ha, hb]))
    ca = torch.bincount(torch.searchsorted(u, ha), minlength=u.numel())
    cb = torch.bincount(torch.searchsorted(u, hb), minlength=u.numel())
    return int(a.shape[0] - torch.minimum(ca, cb).sum().item())


def _ulp32(x: float) -> float:
    """Spacing of float32 values at magnitude x."""
    x = abs(float(np.float32(x)))
    return float(np.spacing(np.float32(x))) if x > 0 else float(np.finfo(np.float32).tiny)


def f32_slack(points, quantizer: int, l2: float) -> float:
    """Float32 resolution of the reference's arithmetic on this cloud (see the module text):
    sqrt(3) * (step * ulp(E / step) + ulp(E) + ulp(M)), E the largest per-axis extent, M the
    largest coordinate magnitude, step the
    quantizer's lattice step (2 l2 / sqrt(5) for the truncated octahedron, 2 l2 / sqrt(3) for
    the cube)."""
    if points.shape[0] == 0:
        return 0.0
    ext = float((points.max(dim=0).values - points.min(dim=0).values).max().item())
    big = float(points.abs().max().item())
    step = float(np.float32(2.0 * np.float32(l2) / np.sqrt(5.0 if quantizer == 1 else 3.0)))
    return float(np.sqrt(3.0) * (step * _ulp32(ext / step) + _ulp32(ext) + _ulp32(big)))


def l2_report(ctx, points, quantizer: int, l2: float, decoded=None) -> dict:
    """Error of every input point against its cell's recovered point, and (with `decoded`, an
    (m, 3) float32 device tensor) how the decoded cloud matches those points.

    points: (n, 3) float32 CUDA tensor.  Returns max_l2_error, over_bound (float compare, as
    main.cpp), f32_slack and over_bound_plus_slack, z_minus1_points, and with `decoded`:
    decoded_points and mismatch (decoded points without an equal recovered input point; equal
    to z_minus1_points in a -rle or -normal container of the truncated octahedron, whose
    wrapped cells decode elsewhere)."""
    import torch
    n = points.shape[0]
    cells = torch.empty((n, 3), dtype=torch.int32, device=points.device)
    rec = torch.empty((n, 3), dtype=torch.float32, device=points.device)
    off = np.zeros(3, np.float32)
    N.check(N.stage_quantize(ctx.handle, C.c_void_p(points.data_ptr()), n, int(quantizer), float(l2),
                             off.ctypes.data_as(C.c_void_p), C.c_void_p(cells.data_ptr())))
    N.check(N.stage_recover(ctx.handle, C.c_void_p(cells.data_ptr()), n, int(quantizer), float(l2),
                            off.ctypes.data_as(C.c_void_p), C.c_void_p(rec.data_ptr())))
    torch.cuda.current_stream(points.device).synchronize()
    d = points - rec
    sq = d * d
    err = torch.sqrt(sq[:, 0] + (sq[:, 1] + sq[:, 2]))
    slack = f32_slack(points, quantizer, l2)
    out = {"max_l2_error": float(err.max().item()) if n else 0.0,
           "over_bound": int((err > l2).sum().item()),
           "f32_slack": slack,
           "over_bound_plus_slack": int((err.double() > l2 + slack).sum().item()),
           "z_minus1_points": int((cells[:, 2] == -1).sum().item()) if quantizer == 1 else 0}
    del cells, err, sq, d
    if decoded is not None:
        out["decoded_points"] = int(decoded.shape[0])
        out["mismatch"] = multiset_mismatch(decoded, rec)
    return out
