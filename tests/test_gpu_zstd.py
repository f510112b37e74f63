"""zstd frames decoded on the GPU (xnyz_zstd_decompress_device): the content equals libzstd's,
for the frames the compressors write and for general data at every level; damaged frames end
with an error status and leave the context usable."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _libzstd():
    from xnyzip_b200 import _native as N
    z = C.CDLL(N.default_zstd_library())
    z.ZSTD_compressBound.restype = C.c_size_t
    z.ZSTD_compressBound.argtypes = [C.c_size_t]
    z.ZSTD_compress.restype = C.c_size_t
    z.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]
    z.ZSTD_isError.restype = C.c_uint
    z.ZSTD_isError.argtypes = [C.c_size_t]
    return z


def _zstd(z, data: bytes, level: int) -> bytes:
    cap = z.ZSTD_compressBound(len(data))
    out = C.create_string_buffer(cap)
    n = z.ZSTD_compress(out, cap, data, len(data), level)
    assert not z.ZSTD_isError(n)
    return out.raw[:n]


def _gpu_decode(ctx, frames, caps):
    """Packs the frames into one device buffer at odd offsets and decodes them in one call."""
    import torch
    offs, pos = [], 0
    for f in frames:
        offs.append(pos + 1)
        pos += len(f) + 3
    src = torch.zeros(max(pos, 1), dtype=torch.uint8)
    for o, f in zip(offs, frames):
        if f:
            src[o:o + len(f)] = torch.frombuffer(bytearray(f), dtype=torch.uint8)
    src = src.cuda()
    out_offs, pos = [], 0
    for c in caps:
        out_offs.append(pos)
        pos += c + 16
    dst = torch.full((max(pos, 1),), 0xA5, dtype=torch.uint8, device="cuda")
    base, dbase = src.data_ptr(), dst.data_ptr()
    lens = ctx.zstd_decompress_device([base + o for o in offs], [len(f) for f in frames],
                                      [dbase + o for o in out_offs], caps)
    host = dst.cpu().numpy().tobytes()
    return lens, [host[o:o + max(int(n), 0)] for o, n in zip(out_offs, lens)], host, out_offs


def test_container_frames(ctx):
    """Frames from the compressors decode to their own pre-zstd containers."""
    from xnyzip_b200 import synthetic as S
    frames, plains = [], []
    for i, (q, l2, hil, rle, n) in enumerate([(1, 0.001, 1, 1, 200000), (0, 0.01, 0, 1, 150000),
                                              (1, 0.05, 1, 0, 120000), (0, 0.1, 1, 0, 3), (1, 0.01, 0, 1, 1)]):
        x = S.terrain(n, seed=30 + i) if i % 2 == 0 else S.with_duplicates(n, seed=40 + i)
        frames.append(ctx.compress(x, q, l2, hil, rle, use_zstd=True))
        plains.append(ctx.compress(x, q, l2, hil, rle, use_zstd=False))
    lens, outs, _, _ = _gpu_decode(ctx, frames, [len(p) for p in plains])
    assert list(lens) == [len(p) for p in plains]
    assert outs == plains


@pytest.mark.parametrize("level", [1, 3, 9, 19])
def test_general_data(ctx, level):
    """Raw, RLE and compressed blocks, 1 and 4 literal streams, FSE and direct Huffman weights,
    predefined, RLE and coded sequence tables, repeat offsets, several blocks per frame."""
    z = _libzstd()
    rng = np.random.default_rng(level)
    data = [b"", b"q", b"hello hello hello world",
            rng.integers(0, 256, 300000, dtype=np.uint8).tobytes(),
            bytes(200000),
            rng.geometric(0.3, 400000).astype(np.uint8).tobytes(),
            b"The quick brown fox jumps over the lazy dog. " * 9000,
            bytes(np.repeat(rng.integers(0, 5, 20000, dtype=np.uint8), rng.integers(1, 40, 20000)))]
    parts = []
    for _ in range(40):
        k, n = int(rng.integers(0, 4)), int(rng.integers(1, 30000))
        parts.append(rng.integers(0, 256, n, dtype=np.uint8).tobytes() if k == 0 else
                     bytes([int(rng.integers(0, 256))]) * n if k == 1 else
                     rng.geometric(float(rng.uniform(0.05, 0.9)), n).astype(np.uint8).tobytes() if k == 2 else
                     parts[int(rng.integers(0, len(parts)))][:n] if parts else b"abc")
    data.append(b"".join(parts))
    frames = [_zstd(z, d, level) for d in data]
    lens, outs, host, offs = _gpu_decode(ctx, frames, [len(d) for d in data])
    assert list(lens) == [len(d) for d in data]
    assert outs == data
    for o, d in zip(offs, data):  # nothing written past the content
        assert host[o + len(d):o + len(d) + 16] == b"\xa5" * 16


def test_damaged_frames(ctx, xnyz):
    """A truncated frame, a frame with a damaged magic number, a capacity one byte short and a
    frame of zeros beside a good one each fail with XNYZ_ERR_BAD_STREAM; the next call on the
    context decodes normally."""
    z = _libzstd()
    data = b"The quick brown fox jumps over the lazy dog. " * 3000
    f = _zstd(z, data, 3)
    flipped = bytearray(f)
    flipped[0] ^= 0x10
    for frames, caps in [([f[:len(f) // 2]], [len(data)]), ([bytes(flipped)], [len(data)]),
                         ([f], [len(data) - 1]), ([f, b"\x00" * 9], [len(data), 64])]:
        with pytest.raises(xnyz.XnyzError):
            _gpu_decode(ctx, frames, caps)
    lens, outs, _, _ = _gpu_decode(ctx, [f], [len(data)])
    assert lens[0] == len(data) and outs[0] == data


def test_too_many_huffman_weights(ctx, xnyz):
    """A frame whose Huffman tree description codes 256 weights (one more than a tree can have)
    fails with XNYZ_ERR_BAD_STREAM, beside a good frame; the context stays usable."""
    from zstd_craft import frame_with_huf_tree, huf_tree_256_weights
    z = _libzstd()
    data = b"0123456789abcdef" * 500
    f = _zstd(z, data, 3)
    bad = frame_with_huf_tree(huf_tree_256_weights())
    with pytest.raises(xnyz.XnyzError) as e:
        _gpu_decode(ctx, [f, bad], [len(data), 256])
    assert e.value.status == 2  # XNYZ_ERR_BAD_STREAM
    lens, outs, _, _ = _gpu_decode(ctx, [f], [len(data)])
    assert lens[0] == len(data) and outs[0] == data


def test_random_frames(ctx):
    """48 seeded frames of mixed random, run, geometric and repeated data (up to ~1.5 MB, levels
    1-19), decoded in one call: every frame equals libzstd's input."""
    z = _libzstd()
    rng = np.random.default_rng(2024)
    data, frames = [], []
    for _ in range(48):
        parts, total, want = [], 0, int(rng.integers(1000, 1_500_000))
        while total < want:
            kind, n = int(rng.integers(0, 4)), int(rng.integers(1, 50000))
            if kind == 0:
                p = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
            elif kind == 1:
                p = bytes([int(rng.integers(0, 256))]) * n
            elif kind == 2:
                p = rng.geometric(float(rng.uniform(0.05, 0.9)), n).astype(np.uint8).tobytes()
            else:
                p = parts[int(rng.integers(0, len(parts)))][:n] if parts else b"abc"
            parts.append(p)
            total += len(p)
        d = b"".join(parts)
        data.append(d)
        frames.append(_zstd(z, d, int(rng.choice([1, 2, 3, 5, 9, 15, 19]))))
    lens, outs, _, _ = _gpu_decode(ctx, frames, [len(d) for d in data])
    assert list(lens) == [len(d) for d in data]
    assert [i for i, (o, d) in enumerate(zip(outs, data)) if o != d] == []
