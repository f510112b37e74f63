"""ctypes access to the oracle (test infrastructure only).

Two libraries live here:
  * ``liboracle.so`` - the project's sequential CPU restatement of the XnYZip path
    (oracle/xnyz_oracle.cpp), built by oracle/build_oracle.sh.  This is the checker used by
    the tests on any machine.
  * ``_ref/libxnyz_ref.so`` - the reference itself, compiled from its own sources by
    oracle/build_ref.sh where the reference is present.  It pins the restatement.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libxnyz_ref.so")
REF_CLI = os.path.join(HERE, "_ref", "xnyzip_ref")

sys.path.insert(0, HERE)
from find_zstd import find_zstd  # noqa: E402

QUANT = {"cube": 0, "to": 1, "adaptive": 2}

_u8p = C.POINTER(C.c_uint8)
_f32p = C.POINTER(C.c_float)


def _buf(arr):
    return arr.ctypes.data_as(C.c_void_p)


class _Lib:
    def __init__(self, path: str, prefix: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        self.p = prefix

    def fn(self, name, argtypes, restype=C.c_int):
        f = getattr(self.lib, self.p + name)
        f.argtypes = argtypes
        f.restype = restype
        return f

    def take(self, ptr, n, dtype=np.uint8):
        if n == 0:
            out = np.zeros(0, dtype=dtype)
        else:
            out = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dtype))),
                                        shape=(n,)).copy()
        self.fn("free", [C.c_void_p], None)(C.cast(ptr, C.c_void_p))
        return out


class Oracle(_Lib):
    """The restatement (liboracle.so)."""

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path, "orc_")
        try:
            self.fn("set_zstd_library", [C.c_char_p])(find_zstd().encode())
        except FileNotFoundError:
            pass

    def compress(self, xyz, quantizer, l2, hilbert, rle, direct_threshold=1024, zstd=True, with_order=False):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        n = xyz.shape[0]
        out, ln = _u8p(), C.c_uint64()
        order = np.zeros(max(n, 1), dtype=np.uint64) if with_order else None
        rc = self.fn("compress", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(_u8p), C.POINTER(C.c_uint64), C.c_void_p])(
            _buf(xyz), n, QUANT.get(quantizer, quantizer), l2, int(hilbert), int(rle), direct_threshold,
            3 if zstd else -1, C.byref(out), C.byref(ln), _buf(order) if with_order else None)
        if rc:
            raise RuntimeError(f"orc_compress failed ({rc})")
        data = self.take(out, ln.value).tobytes()
        return (data, order[: n if n else 0]) if with_order else data

    def fit_profile(self, xyz, quantizer, l2, hilbert, zstd=True):
        """fit_profile (block_compressor.hpp:241-246): (frame, serialized profile)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        out, ln, pr, pl = _u8p(), C.c_uint64(), _u8p(), C.c_uint64()
        rc = self.fn("fit_profile", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int, C.POINTER(_u8p),
                                     C.POINTER(C.c_uint64), C.POINTER(_u8p), C.POINTER(C.c_uint64)])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), 3 if zstd else -1,
            C.byref(out), C.byref(ln), C.byref(pr), C.byref(pl))
        if rc:
            raise RuntimeError(f"orc_fit_profile failed ({rc})")
        return self.take(out, ln.value).tobytes(), self.take(pr, pl.value).tobytes()

    def compress_with_profile(self, xyz, quantizer, l2, hilbert, profile, zstd=True):
        """compress_with_profile (block_compressor.hpp:248-256): the frame."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        pb = np.frombuffer(bytes(profile), dtype=np.uint8)
        out, ln = _u8p(), C.c_uint64()
        rc = self.fn("compress_with_profile", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_void_p,
                                               C.c_uint64, C.c_int, C.POINTER(_u8p), C.POINTER(C.c_uint64)])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), _buf(pb), pb.size,
            3 if zstd else -1, C.byref(out), C.byref(ln))
        if rc:
            raise RuntimeError(f"orc_compress_with_profile failed ({rc})")
        return self.take(out, ln.value).tobytes()

    def decompress(self, buf, quantizer, l2, rle, zstd=True):
        b = np.frombuffer(buf, dtype=np.uint8)
        out, n = _f32p(), C.c_uint64()
        rc = self.fn("decompress", [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_int,
                                    C.POINTER(_f32p), C.POINTER(C.c_uint64)])(
            _buf(b), len(buf), int(zstd), QUANT.get(quantizer, quantizer), l2, int(rle), C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError(f"orc_decompress failed ({rc})")
        return self.take(out, 3 * n.value, np.float32).reshape(-1, 3)

    def quantize(self, xyz, quantizer, l2):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        off = np.zeros(3, np.float32)
        q = np.zeros((xyz.shape[0], 3), np.int32)
        self.fn("quantize", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_void_p, C.c_void_p])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, _buf(off), _buf(q))
        return off, q

    def recover(self, q, quantizer, l2, offset):
        q = np.ascontiguousarray(q, dtype=np.int32).reshape(-1, 3)
        off = np.ascontiguousarray(offset, dtype=np.float32)
        out = np.zeros((q.shape[0], 3), np.float32)
        self.fn("recover", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_void_p, C.c_void_p])(
            _buf(q), q.shape[0], QUANT.get(quantizer, quantizer), l2, _buf(off), _buf(out))
        return out

    def m2h(self, codes, iteration):
        c = np.ascontiguousarray(codes, dtype=np.uint64)
        o = np.zeros_like(c)
        self.fn("m2h", [C.c_void_p, C.c_uint64, C.c_uint, C.c_void_p], None)(_buf(c), c.size, iteration, _buf(o))
        return o

    def h2m(self, codes, iteration):
        c = np.ascontiguousarray(codes, dtype=np.uint64)
        o = np.zeros_like(c)
        self.fn("h2m", [C.c_void_p, C.c_uint64, C.c_uint, C.c_void_p], None)(_buf(c), c.size, iteration, _buf(o))
        return o

    def block_records(self, q, rx, ry, rz, hilbert):
        q = np.ascontiguousarray(q, dtype=np.int32).reshape(-1, 3)
        n = q.shape[0]
        ids = np.zeros(n, np.uint64)
        reid = np.zeros(n, np.uint64)
        self.fn("block_records", [C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                  C.c_void_p])(_buf(q), n, rx, ry, rz, int(hilbert), _buf(ids), _buf(reid))
        return ids, reid

    def _two(self, name, args, argtypes):
        m, ml, e, el = _u8p(), C.c_uint64(), _u8p(), C.c_uint64()
        rc = self.fn(name, argtypes + [C.POINTER(_u8p), C.POINTER(C.c_uint64), C.POINTER(_u8p),
                                       C.POINTER(C.c_uint64)])(*args, C.byref(m), C.byref(ml), C.byref(e), C.byref(el))
        if rc:
            raise ValueError(f"{self.p}{name} failed ({rc})")
        return self.take(m, ml.value).tobytes(), self.take(e, el.value).tobytes()

    def huffman(self, data, kind, force_eg=False):
        dt = {0: np.uint64, 1: np.uint8, 2: np.int32}[kind]
        d = np.ascontiguousarray(data, dtype=dt)
        return self._two("huffman", [kind, _buf(d), d.size, int(force_eg)],
                         [C.c_int, C.c_void_p, C.c_uint64, C.c_int])

    def gr_pack(self, data):
        d = np.ascontiguousarray(data, dtype=np.uint64)
        return self._two("gr_pack", [_buf(d), d.size], [C.c_void_p, C.c_uint64])

    def bitpack(self, data):
        d = np.ascontiguousarray(data, dtype=np.uint64)
        return self._two("bitpack", [_buf(d), d.size], [C.c_void_p, C.c_uint64])


class Reference(Oracle):
    """The reference compiled from its own sources (oracle/_ref/libxnyz_ref.so)."""

    def __init__(self, path: str = REF_SO):
        _Lib.__init__(self, path, "ref_")

    def quiet(self, on=True):
        self.fn("quiet", [C.c_int], None)(int(on))

    def compress(self, xyz, quantizer, l2, hilbert, rle, direct_threshold=1024, with_sorted=False):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        out, ln = _u8p(), C.c_uint64()
        srt = np.zeros_like(xyz) if with_sorted else None
        rc = self.fn("compress", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(_u8p), C.POINTER(C.c_uint64), C.c_void_p])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), int(rle), direct_threshold,
            C.byref(out), C.byref(ln), _buf(srt) if with_sorted else None)
        if rc:
            raise RuntimeError("ref_compress failed")
        data = self.take(out, ln.value).tobytes()
        return (data, srt) if with_sorted else data

    def fit_profile(self, xyz, quantizer, l2, hilbert, direct_threshold=1024):
        """BlockCompressor::fit_profile: (zstd frame, serialize_profile blob)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        out, ln, pr, pl = _u8p(), C.c_uint64(), _u8p(), C.c_uint64()
        rc = self.fn("fit_profile", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int, C.POINTER(_u8p),
                                     C.POINTER(C.c_uint64), C.POINTER(_u8p), C.POINTER(C.c_uint64), C.c_void_p])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), direct_threshold,
            C.byref(out), C.byref(ln), C.byref(pr), C.byref(pl), None)
        if rc:
            raise RuntimeError("ref_fit_profile failed")
        return self.take(out, ln.value).tobytes(), self.take(pr, pl.value).tobytes()

    def compress_with_profile(self, xyz, quantizer, l2, hilbert, profile, direct_threshold=1024):
        """BlockCompressor::compress_with_profile(deserialize_profile(profile)): the frame."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        pb = np.frombuffer(bytes(profile), dtype=np.uint8)
        out, ln = _u8p(), C.c_uint64()
        rc = self.fn("compress_with_profile", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int,
                                               C.c_void_p, C.c_uint64, C.POINTER(_u8p), C.POINTER(C.c_uint64)])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), direct_threshold, _buf(pb),
            pb.size, C.byref(out), C.byref(ln))
        if rc:
            raise RuntimeError("ref_compress_with_profile failed")
        return self.take(out, ln.value).tobytes()

    def decompress(self, buf, quantizer, l2, rle):
        b = np.frombuffer(buf, dtype=np.uint8)
        out, n = _f32p(), C.c_uint64()
        rc = self.fn("decompress", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.POINTER(_f32p),
                                    C.POINTER(C.c_uint64)])(
            _buf(b), len(buf), QUANT.get(quantizer, quantizer), l2, int(rle), C.byref(out), C.byref(n))
        if rc:
            raise RuntimeError("ref_decompress failed")
        return self.take(out, 3 * n.value, np.float32).reshape(-1, 3)

    def encode_cells(self, cells, counts, ranges, offset, hilbert, quantizer="to", l2=0.05):
        """BlockCompressorRLE::encode_cells_with_counts: the zstd frame."""
        cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        off = np.ascontiguousarray(offset, dtype=np.float32)
        out, ln = _u8p(), C.c_uint64()
        rc = self.fn("encode_cells", [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                      C.c_int, C.c_int, C.c_float, C.POINTER(_u8p), C.POINTER(C.c_uint64)])(
            _buf(cells), _buf(counts), cells.shape[0], int(ranges[0]), int(ranges[1]), int(ranges[2]), _buf(off),
            int(hilbert), QUANT.get(quantizer, quantizer), l2, C.byref(out), C.byref(ln))
        if rc:
            raise RuntimeError("ref_encode_cells failed")
        return self.take(out, ln.value).tobytes()

    def decompress_to_cells(self, buf, quantizer="to", l2=0.05):
        """BlockDecompressorRLE::decompress_to_cells: (cells, counts, offset, ranges, hilbert)."""
        b = np.frombuffer(buf, dtype=np.uint8)
        _i32p = C.POINTER(C.c_int32)
        cp, kp, n = _i32p(), _i32p(), C.c_uint64()
        off = np.zeros(3, np.float32)
        rng = np.zeros(3, np.int32)
        hil = C.c_int()
        rc = self.fn("decompress_to_cells", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.POINTER(_i32p),
                                             C.POINTER(_i32p), C.POINTER(C.c_uint64), C.c_void_p, C.c_void_p,
                                             C.POINTER(C.c_int)])(
            _buf(b), len(buf), QUANT.get(quantizer, quantizer), l2, C.byref(cp), C.byref(kp), C.byref(n), _buf(off),
            _buf(rng), C.byref(hil))
        if rc:
            raise RuntimeError("ref_decompress_to_cells failed")
        cells = np.ctypeslib.as_array(cp, shape=(3 * n.value,)).copy().reshape(-1, 3)
        counts = np.ctypeslib.as_array(kp, shape=(n.value,)).copy()
        self.fn("free", [C.c_void_p], None)(C.cast(cp, C.c_void_p))
        self.fn("free", [C.c_void_p], None)(C.cast(kp, C.c_void_p))
        return cells, counts, off, rng, bool(hil.value)

    def expand_cells(self, cells, counts, offset, quantizer="to", l2=0.05):
        """BlockDecompressorRLE::expand_cells_to_points."""
        cells = np.ascontiguousarray(cells, dtype=np.int32).reshape(-1, 3)
        counts = np.ascontiguousarray(counts, dtype=np.int32)
        off = np.ascontiguousarray(offset, dtype=np.float32)
        out, n = _f32p(), C.c_uint64()
        rc = self.fn("expand_cells", [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_int, C.c_float,
                                      C.POINTER(_f32p), C.POINTER(C.c_uint64)])(
            _buf(cells), _buf(counts), cells.shape[0], _buf(off), QUANT.get(quantizer, quantizer), l2, C.byref(out),
            C.byref(n))
        if rc:
            raise RuntimeError("ref_expand_cells failed")
        return self.take(out, 3 * n.value, np.float32).reshape(-1, 3)

    def unzstd(self, buf):
        b = np.frombuffer(buf, dtype=np.uint8)
        out, ln = _u8p(), C.c_uint64()
        rc = self.fn("unzstd", [C.c_void_p, C.c_uint64, C.POINTER(_u8p), C.POINTER(C.c_uint64)])(
            _buf(b), len(buf), C.byref(out), C.byref(ln))
        if rc:
            raise RuntimeError("ref_unzstd failed")
        return self.take(out, ln.value).tobytes()

    def roundtrip_timed(self, xyz, quantizer, l2, hilbert, rle, direct_threshold=1024):
        """Compress + decompress timed by the reference's own Timer: (t_c, t_d, bytes, n)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
        tc, td, cb, nd = C.c_double(), C.c_double(), C.c_uint64(), C.c_uint64()
        rc = self.fn("roundtrip_timed", [C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                         C.POINTER(C.c_uint64)])(
            _buf(xyz), xyz.shape[0], QUANT.get(quantizer, quantizer), l2, int(hilbert), int(rle), direct_threshold,
            C.byref(tc), C.byref(td), C.byref(cb), C.byref(nd))
        if rc:
            raise RuntimeError("ref_roundtrip_timed failed")
        return tc.value, td.value, cb.value, nd.value

    def gr_pack(self, data, kind=0):
        dt = np.uint64 if kind == 0 else np.uint8
        d = np.ascontiguousarray(data, dtype=dt)
        return self._two("gr_pack", [kind, _buf(d), d.size], [C.c_int, C.c_void_p, C.c_uint64])


def available_reference() -> bool:
    return os.path.exists(REF_SO)
