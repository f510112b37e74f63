"""ctypes binding of the C ABI in include/xnyz.h (libxnyz.so, built in-tree).

The library is the product: nothing here computes on the CPU.  Importing fails loudly
when the shared library is missing.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxnyz.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python xnyzip_b200/build.py`")

lib = C.CDLL(LIB_PATH)

STATUS = {
    0: "OK", 1: "INVALID_ARG", 2: "BAD_STREAM", 3: "CUDA", 4: "OOM", 5: "TIMEOUT", 6: "UNSUPPORTED",
    7: "ZSTD", 8: "NO_DEVICE",
}


class XnyzError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"xnyz {STATUS.get(status, status)}: {message}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("quantizer", C.c_int), ("l2_bound", C.c_float), ("hilbert", C.c_int), ("rle", C.c_int),
                ("direct_threshold", C.c_int)]


class CompressInfo(C.Structure):
    _fields_ = [("num_points", C.c_uint64), ("num_units", C.c_uint64), ("num_blocks", C.c_uint64),
                ("num_patches", C.c_uint64), ("container_bytes", C.c_uint64), ("output_bytes", C.c_uint64),
                ("range", C.c_int32 * 3), ("is_direct", C.c_int), ("counts_exp_golomb", C.c_int),
                ("max_l2_error", C.c_double), ("mse", C.c_double), ("gpu_ms", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "range"}
        d["range"] = list(self.range)
        return d


_p = C.c_void_p
_u8pp = C.POINTER(C.POINTER(C.c_uint8))


def _proto(name, argtypes, restype=C.c_int):
    f = getattr(lib, name)
    f.argtypes = argtypes
    f.restype = restype
    return f


create = _proto("xnyz_create", [C.POINTER(_p), C.c_int, _p])
destroy = _proto("xnyz_destroy", [_p])
last_error = _proto("xnyz_last_error", [], C.c_char_p)
version = _proto("xnyz_version", [], C.c_char_p)
set_zstd_library = _proto("xnyz_set_zstd_library", [C.c_char_p])
host_alloc = _proto("xnyz_host_alloc", [C.POINTER(_p), C.c_size_t])
host_free = _proto("xnyz_host_free", [_p])
trim = _proto("xnyz_trim", [_p])
free = _proto("xnyz_free", [_p], None)
compress = _proto("xnyz_compress", [_p, _p, C.c_uint64, C.c_int, C.POINTER(Params), C.c_int, _u8pp,
                                    C.POINTER(C.c_uint64), _p, C.POINTER(CompressInfo)])
fit_profile = _proto("xnyz_fit_profile", [_p, _p, C.c_uint64, C.c_int, C.POINTER(Params), C.c_int, _u8pp,
                                          C.POINTER(C.c_uint64), _p, _u8pp, C.POINTER(C.c_uint64)])
compress_with_profile = _proto("xnyz_compress_with_profile", [_p, _p, C.c_uint64, C.c_int, C.POINTER(Params), _p,
                                                              C.c_uint64, C.c_int, _u8pp, C.POINTER(C.c_uint64), _p])
compress_device = _proto("xnyz_compress_device", [_p, _p, C.c_uint64, C.POINTER(Params), C.POINTER(_p),
                                                  C.POINTER(C.c_uint64), C.POINTER(CompressInfo)])
decompress = _proto("xnyz_decompress", [_p, _p, C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_int,
                                        C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_uint64)])
decompress_into = _proto("xnyz_decompress_into", [_p, _p, C.c_uint64, C.c_int, C.c_int, C.c_float, C.c_int, _p,
                                                  C.c_uint64, C.POINTER(C.c_uint64)])
decompress_device = _proto("xnyz_decompress_device", [_p, _p, C.c_uint64, C.c_int, C.c_float, C.c_int,
                                                      C.POINTER(_p), C.POINTER(C.c_uint64)])
stage_quantize = _proto("xnyz_stage_quantize", [_p, _p, C.c_uint64, C.c_int, C.c_float, _p, _p])
stage_recover = _proto("xnyz_stage_recover", [_p, _p, C.c_uint64, C.c_int, C.c_float, _p, _p])
stage_hilbert = _proto("xnyz_stage_hilbert", [_p, _p, C.c_uint64, C.c_uint, C.c_int, _p])
stage_sort = _proto("xnyz_stage_sort", [_p, _p, _p, C.c_uint64, C.c_int])
sort_noalloc = _proto("xnyz_sort_noalloc", [_p, _p, C.c_uint64, C.c_int, _p])
batch_create = _proto("xnyz_batch_create", [C.POINTER(_p), C.c_int, C.c_int])
batch_destroy = _proto("xnyz_batch_destroy", [_p])
batch_workers = _proto("xnyz_batch_workers", [_p])
batch_compress = _proto("xnyz_batch_compress", [_p, C.c_uint64, _p, _p, C.c_int, _p, C.c_int, _p, _p, _p])
batch_decompress = _proto("xnyz_batch_decompress", [_p, C.c_uint64, _p, _p, C.c_int, _p, _p, _p, _p, _p, _p, _p])
batch_roundtrip = _proto("xnyz_batch_roundtrip", [_p, C.c_uint64, _p, _p, _p, _p, _p, _p, _p])
zstd_decompress_device = _proto("xnyz_zstd_decompress_device", [_p, C.c_uint64, _p, _p, _p, _p, _p])
profile = _proto("xnyz_profile", [_p, C.c_int])
profile_read = _proto("xnyz_profile_read", [_p, C.c_char_p, C.c_uint64, C.POINTER(C.c_uint64)])
host_hilbert = _proto("xnyz_host_hilbert", [_p, C.c_uint64, C.c_uint, C.c_int, _p])
host_codebook = _proto("xnyz_host_codebook", [C.c_int, C.c_int, _p, _p, _p, C.c_uint64, C.c_uint64, _p,
                                              C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_int)])

class BlockInfo(C.Structure):
    _fields_ = [("values", C.c_uint64), ("blocks", C.c_uint64), ("payload_bits", C.c_uint64),
                ("fallback_blocks", C.c_uint64), ("mode", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


set_block_mode = _proto("xnyz_set_block_mode", [_p, C.c_int])
set_model = _proto("xnyz_set_model", [_p, _p, C.c_uint64, C.c_float])
model_param_count = _proto("xnyz_model_param_count", [], C.c_uint64)
last_block_info = _proto("xnyz_last_block_info", [_p, C.POINTER(BlockInfo)])
batch_set_block_mode = _proto("xnyz_batch_set_block_mode", [_p, C.c_int])
stage_repos = _proto("xnyz_stage_repos", [_p, _p, C.c_uint64, C.POINTER(Params), _p, C.c_uint64,
                                          C.POINTER(C.c_uint64)])
block_features = _proto("xnyz_block_features", [_p, C.c_uint64, _p, _p])
block_search = _proto("xnyz_block_search", [_p, C.c_uint64, _p, _p, _p, _p])
block_cost = _proto("xnyz_block_cost", [_p, C.c_uint64, _p, _p, _p, _p])
mlp_forward = _proto("xnyz_mlp_forward", [_p, _p, C.c_uint64, _p, _p, _p, _p, _p])
mlp_gather_floats = _proto("xnyz_mlp_gather_floats", [C.c_uint64], C.c_uint64)
mlp_train_batch = _proto("xnyz_mlp_train_batch", [_p, _p, _p, _p, _p, C.c_uint64, C.c_uint64, C.c_float, _p, _p, _p,
                                                  _p])
mlp_adam = _proto("xnyz_mlp_adam", [_p, _p, _p, _p, C.c_float, C.c_int, _p])

batch_roundtrip_device = _proto("xnyz_batch_roundtrip_device", [_p, C.c_uint64, _p, _p, _p, _p, _p, _p])
batch_autotune = _proto("xnyz_batch_autotune", [_p, C.c_uint64, _p, _p, _p, _p])

encode_cells = _proto("xnyz_encode_cells", [_p, _p, _p, C.c_uint64, C.c_int, _p, _p, C.c_int, C.c_int, _u8pp,
                                            C.POINTER(C.c_uint64)])
decompress_to_cells = _proto("xnyz_decompress_to_cells", [_p, _p, C.c_uint64, C.c_int, C.POINTER(C.POINTER(C.c_int32)),
                                                          C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.c_uint64), _p,
                                                          _p, C.POINTER(C.c_int)])
expand_cells = _proto("xnyz_expand_cells", [_p, _p, _p, C.c_uint64, C.c_int, C.c_float, _p,
                                            C.POINTER(C.POINTER(C.c_float)), C.POINTER(C.c_uint64)])

BLOCKS_OFF, BLOCKS_EXHAUSTIVE, BLOCKS_LEARNED, BLOCKS_GLOBAL = 0, 1, 2, 3

# Every symbol include/xnyz.h declares (checked by the tests).
EXPORTED = [
    "xnyz_create", "xnyz_destroy", "xnyz_last_error", "xnyz_version", "xnyz_set_zstd_library", "xnyz_host_alloc",
    "xnyz_host_free", "xnyz_trim", "xnyz_compress", "xnyz_compress_device", "xnyz_decompress",
    "xnyz_decompress_device", "xnyz_free", "xnyz_stage_quantize", "xnyz_stage_recover", "xnyz_stage_hilbert",
    "xnyz_stage_sort", "xnyz_host_hilbert", "xnyz_host_codebook", "xnyz_profile", "xnyz_profile_read", "xnyz_fit_profile", "xnyz_compress_with_profile", "xnyz_sort_noalloc", "xnyz_decompress_into",
    "xnyz_batch_create", "xnyz_batch_destroy", "xnyz_batch_workers", "xnyz_batch_compress", "xnyz_batch_decompress", "xnyz_batch_roundtrip", "xnyz_zstd_decompress_device",
    "xnyz_set_block_mode", "xnyz_set_model", "xnyz_model_param_count", "xnyz_last_block_info",
    "xnyz_batch_set_block_mode", "xnyz_stage_repos", "xnyz_block_features", "xnyz_block_search", "xnyz_block_cost",
    "xnyz_mlp_forward", "xnyz_mlp_gather_floats", "xnyz_mlp_train_batch", "xnyz_mlp_adam",
    "xnyz_batch_roundtrip_device", "xnyz_batch_autotune", "xnyz_encode_cells", "xnyz_decompress_to_cells",
    "xnyz_expand_cells",
]


def check(status: int):
    if status != 0:
        raise XnyzError(status, last_error().decode(errors="replace"))


def default_zstd_library() -> str:
    """libzstd 1.5.7 bundled on this image (Pillow's wheel), or '' if absent."""
    env = os.environ.get("XNYZ_ZSTD_LIBRARY")
    if env:
        return env
    for root in sorted({sysconfig.get_paths()["purelib"], sysconfig.get_paths()["platlib"]}):
        hits = sorted(glob.glob(os.path.join(root, "pillow.libs", "libzstd-*.so.1.5.7")))
        if hits:
            return hits[0]
    return ""


_zstd = default_zstd_library()
if _zstd:
    set_zstd_library(_zstd.encode())
