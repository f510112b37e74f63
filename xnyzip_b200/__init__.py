"""XnYZip compress/decompress path on B200 (sm_100a).

Python mirror of the reference's composer interface (composer/block_compressor.hpp,
composer/block_compressor_rle.hpp, composer/block_decompressor.hpp,
composer/block_decompressor_rle.hpp, composer/utils.hpp) over the C ABI of libxnyz.so:

    BlockCompressor(QUANTIZER_TYPE.TRUNCATED_OCTAHEDRON, 0.05).compress(points, curve_type)
    BlockDecompressor(QUANTIZER_TYPE.TRUNCATED_OCTAHEDRON, 0.05).decompress(data)

`points` is an (n, 3) float32 array (numpy on the host, or a CUDA torch tensor); the
result of compress() is the zstd frame the reference returns, byte for byte.  Every compute
stage runs in hand-written CUDA kernels; the module raises ImportError if the library is
not built.
"""
from __future__ import annotations

import ctypes as C
import enum
import weakref

import numpy as np

from . import _native as N
from ._native import CompressInfo, Params, XnyzError

__all__ = ["QUANTIZER_TYPE", "Context", "Batch", "BlockCompressor", "BlockCompressorRLE", "BlockDecompressor",
           "BlockDecompressorRLE", "XnyzError", "CompressInfo", "default_context"]


class QUANTIZER_TYPE(enum.IntEnum):
    """composer/utils.hpp:55-59."""
    CUBE = 0
    TRUNCATED_OCTAHEDRON = 1
    ADAPTIVE = 2


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class Context:
    """One device, one CUDA stream, one cached workspace (an xnyz_ctx)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        h = C.c_void_p()
        N.check(N.create(C.byref(h), device, C.c_void_p(stream) if stream else None))
        self.handle = h
        self.device = device
        self.last_info = CompressInfo()

    def close(self):
        if self.handle:
            N.destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- profiling --------------------------------------------------------------------
    def profile(self, enable: bool = True):
        N.check(N.profile(self.handle, int(enable)))

    def profile_read(self) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        ln = C.c_uint64()
        N.check(N.profile_read(self.handle, buf, len(buf), C.byref(ln)))
        return json.loads(buf.value.decode())

    # -- whole path -------------------------------------------------------------------
    def compress(self, points, quantizer: int, l2: float, hilbert: bool, rle: bool, direct_threshold: int = 1024,
                 use_zstd: bool = True, want_order: bool = False):
        prm = Params(int(quantizer), float(l2), int(bool(hilbert)), int(bool(rle)), int(direct_threshold))
        out = C.POINTER(C.c_uint8)()
        ln = C.c_uint64()
        info = CompressInfo()
        if _is_torch_cuda(points):
            pts = points.contiguous()
            n = pts.numel() // 3
            ptr, on_dev = C.c_void_p(pts.data_ptr()), 1
        else:
            pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
            n = pts.shape[0]
            ptr, on_dev = pts.ctypes.data_as(C.c_void_p), 0
        order = np.zeros(max(n, 1), dtype=np.uint64) if want_order else None
        N.check(N.compress(self.handle, ptr, n, on_dev, C.byref(prm), int(use_zstd), C.byref(out), C.byref(ln),
                           order.ctypes.data_as(C.c_void_p) if want_order else None, C.byref(info)))
        try:
            data = C.string_at(out, ln.value)
        finally:
            N.free(C.cast(out, C.c_void_p))
        self.last_info = info
        return (data, order[:n]) if want_order else data

    @staticmethod
    def _host_points(points):
        if _is_torch_cuda(points):
            pts = points.contiguous()
            return pts, pts.numel() // 3, C.c_void_p(pts.data_ptr()), 1
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        return pts, pts.shape[0], pts.ctypes.data_as(C.c_void_p), 0

    def fit_profile(self, points, quantizer: int, l2: float, hilbert: bool, use_zstd: bool = True,
                    want_order: bool = False):
        """BlockCompressor::fit_profile (xnyz_fit_profile): (frame, profile[, order]); the
        profile is the serialize_profile blob of the complete codebooks."""
        prm = Params(int(quantizer), float(l2), int(bool(hilbert)), 0, 1024)
        pts, n, ptr, on_dev = self._host_points(points)
        out, ln = C.POINTER(C.c_uint8)(), C.c_uint64()
        prof, pl = C.POINTER(C.c_uint8)(), C.c_uint64()
        order = np.zeros(max(n, 1), dtype=np.uint64) if want_order else None
        N.check(N.fit_profile(self.handle, ptr, n, on_dev, C.byref(prm), int(use_zstd), C.byref(out), C.byref(ln),
                              order.ctypes.data_as(C.c_void_p) if want_order else None, C.byref(prof), C.byref(pl)))
        try:
            data, blob = C.string_at(out, ln.value), C.string_at(prof, pl.value)
        finally:
            N.free(C.cast(out, C.c_void_p))
            N.free(C.cast(prof, C.c_void_p))
        return (data, blob, order[:n]) if want_order else (data, blob)

    def compress_with_profile(self, points, quantizer: int, l2: float, hilbert: bool, profile: bytes,
                              use_zstd: bool = True, want_order: bool = False):
        """BlockCompressor::compress_with_profile (xnyz_compress_with_profile)."""
        prm = Params(int(quantizer), float(l2), int(bool(hilbert)), 0, 1024)
        pts, n, ptr, on_dev = self._host_points(points)
        blob = np.frombuffer(bytes(profile), dtype=np.uint8)
        out, ln = C.POINTER(C.c_uint8)(), C.c_uint64()
        order = np.zeros(max(n, 1), dtype=np.uint64) if want_order else None
        N.check(N.compress_with_profile(self.handle, ptr, n, on_dev, C.byref(prm),
                                        blob.ctypes.data_as(C.c_void_p) if blob.size else None, blob.size,
                                        int(use_zstd), C.byref(out), C.byref(ln),
                                        order.ctypes.data_as(C.c_void_p) if want_order else None))
        try:
            data = C.string_at(out, ln.value)
        finally:
            N.free(C.cast(out, C.c_void_p))
        return (data, order[:n]) if want_order else data

    def decompress(self, data: bytes, quantizer: int, l2: float, rle: bool, is_zstd: bool = True,
                   out: np.ndarray | None = None) -> np.ndarray:
        """Decoded points as an (n, 3) float32 array.  With `out` (e.g. a view of pinned
        memory) the points are copied straight into it and a view of its first n rows is
        returned."""
        buf = np.frombuffer(data, dtype=np.uint8)
        if out is not None:
            o = out.reshape(-1, 3)
            if o.dtype != np.float32 or not o.flags.c_contiguous:
                raise ValueError("out must be a C-contiguous float32 array")
            n = C.c_uint64()
            N.check(N.decompress_into(self.handle, buf.ctypes.data_as(C.c_void_p), len(data), int(is_zstd),
                                      int(quantizer), float(l2), int(bool(rle)), o.ctypes.data_as(C.c_void_p),
                                      o.shape[0], C.byref(n)))
            return o[: n.value]
        out = C.POINTER(C.c_float)()
        n = C.c_uint64()
        N.check(N.decompress(self.handle, buf.ctypes.data_as(C.c_void_p), len(data), int(is_zstd), int(quantizer),
                             float(l2), int(bool(rle)), C.byref(out), C.byref(n)))
        try:
            arr = np.ctypeslib.as_array(out, shape=(3 * n.value,)).copy() if n.value else np.zeros(0, np.float32)
        finally:
            N.free(C.cast(out, C.c_void_p))
        return arr.reshape(-1, 3)

    def compress_device(self, dev_ptr: int, n: int, quantizer: int, l2: float, hilbert: bool, rle: bool,
                        direct_threshold: int = 1024):
        """Device points -> device container (pointer, length) owned by the context."""
        prm = Params(int(quantizer), float(l2), int(bool(hilbert)), int(bool(rle)), int(direct_threshold))
        p = C.c_void_p()
        ln = C.c_uint64()
        info = CompressInfo()
        N.check(N.compress_device(self.handle, C.c_void_p(dev_ptr), n, C.byref(prm), C.byref(p), C.byref(ln),
                                  C.byref(info)))
        self.last_info = info
        return p.value, ln.value

    # -- extended container (block parameters of the repos / SFC-delta stream) ---------
    def set_block_mode(self, mode: int):
        """0 reference container, 1 exhaustive, 2 learned, 3 one global pair (N.BLOCKS_*)."""
        N.check(N.set_block_mode(self.handle, int(mode)))

    def set_model(self, params: np.ndarray, fallback_confidence: float = 0.5):
        prm = np.ascontiguousarray(params, dtype=np.float32).ravel()
        N.check(N.set_model(self.handle, prm.ctypes.data_as(C.c_void_p), prm.size, float(fallback_confidence)))

    def block_info(self) -> dict:
        bi = N.BlockInfo()
        N.check(N.last_block_info(self.handle, C.byref(bi)))
        return bi.as_dict()

    def stage_repos(self, dev_ptr: int, n: int, quantizer: int, l2: float, hilbert: bool, rle: bool, out_ptr: int,
                    cap: int, direct_threshold: int = 1024) -> int:
        """Repos / SFC-delta value of every unit (device u64 array at out_ptr); returns the count."""
        prm = Params(int(quantizer), float(l2), int(bool(hilbert)), int(bool(rle)), int(direct_threshold))
        cnt = C.c_uint64()
        N.check(N.stage_repos(self.handle, C.c_void_p(dev_ptr), n, C.byref(prm), C.c_void_p(out_ptr), cap,
                              C.byref(cnt)))
        return cnt.value

    # -- distributed-RLE cell tables --------------------------------------------------
    def encode_cells(self, cells, counts, ranges, offset, hilbert: bool, use_zstd: bool = True) -> bytes:
        """encode_cells_with_counts: int32 (n, 3) cells, int32 counts, global ranges / offset."""
        cl = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        ct = np.ascontiguousarray(counts, dtype=np.int32)
        rg = np.ascontiguousarray(ranges, dtype=np.int32)
        of = np.ascontiguousarray(offset, dtype=np.float32)
        out = C.POINTER(C.c_uint8)()
        ln = C.c_uint64()
        N.check(N.encode_cells(self.handle, cl.ctypes.data_as(C.c_void_p), ct.ctypes.data_as(C.c_void_p), cl.shape[0],
                               0, rg.ctypes.data_as(C.c_void_p), of.ctypes.data_as(C.c_void_p), int(bool(hilbert)),
                               int(use_zstd), C.byref(out), C.byref(ln)))
        try:
            return C.string_at(out, ln.value)
        finally:
            N.free(C.cast(out, C.c_void_p))

    def decompress_to_cells(self, data: bytes, is_zstd: bool = True):
        """(cells (n, 3) int32, counts int32, offset float32[3], ranges int32[3], hilbert)."""
        cp, kp = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)()
        n = C.c_uint64()
        of = np.zeros(3, np.float32)
        rg = np.zeros(3, np.int32)
        hil = C.c_int()
        N.check(N.decompress_to_cells(self.handle, data, len(data), int(is_zstd), C.byref(cp), C.byref(kp), C.byref(n),
                                      of.ctypes.data_as(C.c_void_p), rg.ctypes.data_as(C.c_void_p), C.byref(hil)))
        try:
            cells = np.ctypeslib.as_array(cp, shape=(3 * n.value,)).copy().reshape(-1, 3) if n.value else \
                np.zeros((0, 3), np.int32)
            counts = np.ctypeslib.as_array(kp, shape=(n.value,)).copy() if n.value else np.zeros(0, np.int32)
        finally:
            N.free(C.cast(cp, C.c_void_p))
            N.free(C.cast(kp, C.c_void_p))
        return cells, counts, of, rg, bool(hil.value)

    def expand_cells(self, cells, counts, offset, quantizer: int, l2: float) -> np.ndarray:
        """expand_cells_to_points: points (sum(counts), 3) float32."""
        cl = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        ct = np.ascontiguousarray(counts, dtype=np.int32)
        of = np.ascontiguousarray(offset, dtype=np.float32)
        out = C.POINTER(C.c_float)()
        n = C.c_uint64()
        N.check(N.expand_cells(self.handle, cl.ctypes.data_as(C.c_void_p), ct.ctypes.data_as(C.c_void_p), cl.shape[0],
                               int(quantizer), float(l2), of.ctypes.data_as(C.c_void_p), C.byref(out), C.byref(n)))
        try:
            return np.ctypeslib.as_array(out, shape=(3 * n.value,)).copy().reshape(-1, 3) if n.value else \
                np.zeros((0, 3), np.float32)
        finally:
            N.free(C.cast(out, C.c_void_p))

    def decompress_device(self, dev_ptr: int, length: int, quantizer: int, l2: float, rle: bool):
        """Device container -> (device pointer to 3*n floats owned by the context, n)."""
        p = C.c_void_p()
        n = C.c_uint64()
        N.check(N.decompress_device(self.handle, C.c_void_p(dev_ptr), length, int(quantizer), float(l2),
                                    int(bool(rle)), C.byref(p), C.byref(n)))
        return p.value, n.value

    def zstd_decompress_device(self, frame_ptrs, frame_lens, out_ptrs, out_caps) -> np.ndarray:
        """Decodes zstd frames in device memory on the GPU (xnyz_zstd_decompress_device); returns
        the content sizes as int64."""
        k = len(frame_ptrs)
        arrs = [np.ascontiguousarray(a, dtype=np.uint64) for a in (frame_ptrs, frame_lens, out_ptrs, out_caps)]
        if any(a.shape != (k,) for a in arrs):
            raise ValueError("one pointer, length, output and capacity per frame")
        out = np.zeros(k, np.int64)
        N.check(N.zstd_decompress_device(self.handle, k, *(a.ctypes.data_as(C.c_void_p) for a in arrs),
                                         out.ctypes.data_as(C.c_void_p)))
        return out


class Batch:
    """Many independent clouds at once (xnyz_batch_*): a pool of worker threads, each with
    its own context and stream; outputs are identical to per-cloud Context calls."""

    def __init__(self, device: int = 0, workers: int = 0):
        h = C.c_void_p()
        N.check(N.batch_create(C.byref(h), device, int(workers)))
        self.handle = h
        self.workers = N.batch_workers(h)

    def close(self):
        if self.handle:
            N.batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compress(self, clouds, params, use_zstd: bool = True, item_status: np.ndarray | None = None,
                 as_bytes: bool = True):
        """clouds: sequence of (n_i, 3) float32 host arrays; params: sequence of
        (quantizer, l2, hilbert, rle[, direct_threshold]).  Returns a list of frames: bytes,
        or (as_bytes=False) uint8 arrays over the library's buffers, freed with the arrays."""
        k = len(clouds)
        arrs = [np.ascontiguousarray(c, dtype=np.float32).reshape(-1, 3) for c in clouds]
        ptrs = (C.c_void_p * k)(*[a.ctypes.data for a in arrs])
        ns = (C.c_uint64 * k)(*[a.shape[0] for a in arrs])
        prm = (Params * k)(*[Params(int(p[0]), float(p[1]), int(bool(p[2])), int(bool(p[3])),
                                    int(p[4]) if len(p) > 4 else 1024) for p in params])
        outs = (C.c_void_p * k)()
        lens = (C.c_uint64 * k)()
        sts = (C.c_int * k)()
        s = N.batch_compress(self.handle, k, ptrs, ns, 0, prm, int(use_zstd), outs, lens, sts)
        frames = []
        for i in range(k):
            if not outs[i]:
                frames.append(None)
            elif as_bytes:
                frames.append(C.string_at(outs[i], lens[i]))
                N.free(outs[i])
            else:
                buf = (C.c_uint8 * max(1, lens[i])).from_address(outs[i])
                weakref.finalize(buf, N.free, outs[i])
                frames.append(np.frombuffer(buf, np.uint8, count=lens[i]))
        if item_status is not None:
            item_status[:k] = list(sts)
        N.check(s)
        return frames

    def roundtrip(self, clouds, params, outs, as_bytes: bool = False):
        """xnyz_batch_roundtrip: every cloud compressed to its zstd frame and decompressed into
        outs[i] on the same worker.  params: (quantizer, l2, hilbert, rle[, direct_threshold]);
        outs: C-contiguous float32 arrays of n_i points.  Returns the frames (uint8 arrays over
        the library's buffers, or bytes)."""
        k = len(clouds)
        arrs = [np.ascontiguousarray(c, dtype=np.float32).reshape(-1, 3) for c in clouds]
        os_ = [o.reshape(-1, 3) for o in outs]
        for a, o in zip(arrs, os_):
            if o.dtype != np.float32 or not o.flags.c_contiguous or o.shape[0] < a.shape[0]:
                raise ValueError("outputs must be C-contiguous float32 arrays of n points")
        ptrs = (C.c_void_p * k)(*[a.ctypes.data for a in arrs])
        ns = (C.c_uint64 * k)(*[a.shape[0] for a in arrs])
        prm = (Params * k)(*[Params(int(p[0]), float(p[1]), int(bool(p[2])), int(bool(p[3])),
                                    int(p[4]) if len(p) > 4 else 1024) for p in params])
        frames_p = (C.c_void_p * k)()
        lens = (C.c_uint64 * k)()
        optr = (C.c_void_p * k)(*[o.ctypes.data for o in os_])
        s = N.batch_roundtrip(self.handle, k, ptrs, ns, prm, frames_p, lens, optr, None)
        frames = []
        for i in range(k):
            if not frames_p[i]:
                frames.append(None)
            elif as_bytes:
                frames.append(C.string_at(frames_p[i], lens[i]))
                N.free(frames_p[i])
            else:
                buf = (C.c_uint8 * max(1, lens[i])).from_address(frames_p[i])
                weakref.finalize(buf, N.free, frames_p[i])
                frames.append(np.frombuffer(buf, np.uint8, count=lens[i]))
        N.check(s)
        return frames

    def set_block_mode(self, mode: int):
        N.check(N.batch_set_block_mode(self.handle, int(mode)))

    @staticmethod
    def _device_args(ptrs, ns, params):
        k = len(ptrs)
        xs = (C.c_void_p * k)(*[C.c_void_p(p) for p in ptrs])
        nn = np.ascontiguousarray(ns, dtype=np.uint64)
        prm = (Params * k)(*[Params(int(q), float(l2), int(bool(h)), int(bool(r)), int(dt)) for q, l2, h, r, dt in params])
        return k, xs, nn, prm

    def roundtrip_device(self, ptrs, ns, params):
        """Device points (pointers, counts, (quantizer, l2, hilbert, rle, direct_threshold)) ->
        (container bytes, decoded point counts) of each cloud; containers stay in HBM."""
        k, xs, nn, prm = self._device_args(ptrs, ns, params)
        ln = np.zeros(k, np.uint64)
        no = np.zeros(k, np.uint64)
        N.check(N.batch_roundtrip_device(self.handle, k, xs, nn.ctypes.data_as(C.c_void_p), prm,
                                         ln.ctypes.data_as(C.c_void_p), no.ctypes.data_as(C.c_void_p), None))
        return ln, no

    def autotune(self, ptrs, ns, params):
        """Workers per size class, chosen by timing the device round trip on samples."""
        k, xs, nn, prm = self._device_args(ptrs, ns, params)
        w = np.zeros(6, np.int32)
        N.check(N.batch_autotune(self.handle, k, xs, nn.ctypes.data_as(C.c_void_p), prm, w.ctypes.data_as(C.c_void_p)))
        return w.tolist()

    def decompress(self, frames, params, outs, is_zstd: bool = True):
        """frames: sequence of bytes; params: (quantizer, l2, rle) per frame; outs: C-contiguous
        float32 arrays (e.g. views of pinned memory) receiving the points.  Returns the point
        counts."""
        k = len(frames)
        bufs = [f if isinstance(f, np.ndarray) else np.frombuffer(f, dtype=np.uint8) for f in frames]
        ins = (C.c_void_p * k)(*[b.ctypes.data for b in bufs])
        lens = (C.c_uint64 * k)(*[len(f) for f in frames])
        qs = (C.c_int * k)(*[int(p[0]) for p in params])
        l2s = (C.c_float * k)(*[float(p[1]) for p in params])
        rles = (C.c_int * k)(*[int(bool(p[2])) for p in params])
        os_ = [o.reshape(-1, 3) for o in outs]
        for o in os_:
            if o.dtype != np.float32 or not o.flags.c_contiguous:
                raise ValueError("outputs must be C-contiguous float32 arrays")
        optr = (C.c_void_p * k)(*[o.ctypes.data for o in os_])
        caps = (C.c_uint64 * k)(*[o.shape[0] for o in os_])
        ns = (C.c_uint64 * k)()
        sts = (C.c_int * k)()
        N.check(N.batch_decompress(self.handle, k, ins, lens, int(is_zstd), qs, l2s, rles, optr, caps, ns, sts))
        return list(ns)


_default: Context | None = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


class _CompressorBase:
    _rle = False

    def __init__(self, quantizer_type: QUANTIZER_TYPE, l2_bound: float, is_debugging: bool = False,
                 direct_threshold: int = 1024, context: Context | None = None):
        self.quantizer = int(QUANTIZER_TYPE(quantizer_type))
        self.l2_bound = float(np.float32(l2_bound))
        self.direct_threshold = int(direct_threshold)
        self.ctx = context

    def compress(self, points, curve_type: bool) -> bytes:
        """Returns the zstd frame.  For -normal, reorders a numpy `points` array in place into
        the container's point order, as the reference does with its argument
        (block_compressor.hpp:141-144, 105-108)."""
        ctx = self.ctx or default_context()
        inplace = (not self._rle) and isinstance(points, np.ndarray)
        res = ctx.compress(points, self.quantizer, self.l2_bound, bool(curve_type), self._rle, self.direct_threshold,
                           use_zstd=True, want_order=inplace)
        if inplace:
            data, order = res
            view = points.reshape(-1, 3)
            view[:] = view[order.astype(np.int64)]
            return data
        return res


class BlockCompressor(_CompressorBase):
    """composer/block_compressor.hpp:31-39 (-normal container)."""
    _rle = False

    def _reorder(self, points, order):
        if isinstance(points, np.ndarray):
            view = points.reshape(-1, 3)
            view[:] = view[order.astype(np.int64)]

    def fit_profile(self, points, curve_type: bool):
        """block_compressor.hpp:241-246: (zstd frame, profile); reorders a numpy `points`
        array into container order like compress()."""
        ctx = self.ctx or default_context()
        data, prof, order = ctx.fit_profile(points, self.quantizer, self.l2_bound, bool(curve_type), want_order=True)
        self._reorder(points, order)
        return data, prof

    def compress_with_profile(self, points, curve_type: bool, profile: bytes) -> bytes:
        """block_compressor.hpp:248-256."""
        ctx = self.ctx or default_context()
        data, order = ctx.compress_with_profile(points, self.quantizer, self.l2_bound, bool(curve_type), profile,
                                                want_order=True)
        self._reorder(points, order)
        return data


class BlockCompressorRLE(_CompressorBase):
    """composer/block_compressor_rle.hpp:30-38 (-rle container)."""
    _rle = True


class _DecompressorBase:
    _rle = False

    def __init__(self, quantizer_type: QUANTIZER_TYPE, l2_bound: float, is_debugging: bool = False,
                 context: Context | None = None):
        self.quantizer = int(QUANTIZER_TYPE(quantizer_type))
        self.l2_bound = float(np.float32(l2_bound))
        self.ctx = context

    def decompress(self, compressed_data: bytes) -> np.ndarray:
        ctx = self.ctx or default_context()
        return ctx.decompress(compressed_data, self.quantizer, self.l2_bound, self._rle, is_zstd=True)


class BlockDecompressor(_DecompressorBase):
    """composer/block_decompressor.hpp:25-31."""
    _rle = False


class BlockDecompressorRLE(_DecompressorBase):
    """composer/block_decompressor_rle.hpp:26-32."""
    _rle = True
