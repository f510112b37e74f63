"""The GPU zstd decoder's source (xnyzip_b200/csrc/zstd_dec.cuh) compiled for the host: with a
one-thread team, and with 32 threads standing in for the lanes of a warp (a std::barrier for the
team barrier; collectives through relaxed atomics, so that like warp shuffles they order no other
memory).  Both must return libzstd's content, the 32 threads must agree, and damaged frames must
end with a negative code."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "xnyzip_b200", "csrc", "zstd_dec.cuh")

HARNESS = r"""
#include "zstd_dec.cuh"
#include <algorithm>
#include <atomic>
#include <barrier>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
using ull = unsigned long long;
struct Shared {
    std::barrier<> bar{32};
    std::atomic<ull> w[32];
    std::atomic<unsigned> arrive{0}, gen{0};
};
struct ThreadTeam {
    int rank;
    static constexpr int size = 32;
    Shared* sh;
    void sync() const { sh->bar.arrive_and_wait(); }
    void xbar() const {
        const unsigned g = sh->gen.load(std::memory_order_relaxed);
        if (sh->arrive.fetch_add(1, std::memory_order_relaxed) == 31) {
            sh->arrive.store(0, std::memory_order_relaxed);
            sh->gen.store(g + 1, std::memory_order_relaxed);
        } else {
            while (sh->gen.load(std::memory_order_relaxed) == g) std::this_thread::yield();
        }
    }
    ull get(int k) const { return sh->w[k].load(std::memory_order_relaxed); }
    void put(ull v) const { sh->w[rank].store(v, std::memory_order_relaxed); xbar(); }
    int min(int v) const {
        put((ull)(long long)v);
        long long m = v;
        for (int k = 0; k < 32; ++k) m = std::min(m, (long long)get(k));
        xbar();
        return (int)m;
    }
    int bcast0(int v) const { put((ull)(long long)v); const int r = (int)(long long)get(0); xbar(); return r; }
};
static xnyz::zd::Workspace* fresh_ws() {
    auto* ws = static_cast<xnyz::zd::Workspace*>(std::malloc(sizeof(xnyz::zd::Workspace)));
    std::memset(ws, 0xA7, sizeof(*ws));  // stale contents must not matter
    return ws;
}
extern "C" long long zd_solo(const unsigned char* s, ull len, unsigned char* d, ull cap) {
    auto* ws = fresh_ws();
    const long long r = xnyz::zd::decode_frame(s, len, d, cap, *ws, xnyz::zd::SoloTeam{});
    std::free(ws);
    return r;
}
extern "C" long long zd_team(const unsigned char* s, ull len, unsigned char* d, ull cap) {
    auto* ws = fresh_ws();
    Shared sh;
    long long res[32];
    std::vector<std::thread> th;
    for (int r = 0; r < 32; ++r)
        th.emplace_back([&, r] { res[r] = xnyz::zd::decode_frame(s, len, d, cap, *ws, ThreadTeam{r, &sh}); });
    for (auto& t : th) t.join();
    std::free(ws);
    for (int r = 1; r < 32; ++r)
        if (res[r] != res[0]) return -100;  // the lanes disagree
    return res[0];
}
"""


@pytest.fixture(scope="module")
def zd(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("zd")
    shutil.copy(HEADER, d / "zstd_dec.cuh")
    (d / "h.cpp").write_text(HARNESS)
    lib = d / "libzd.so"
    subprocess.run([cxx, "-O2", "-std=c++20", "-shared", "-fPIC", "-pthread", str(d / "h.cpp"), "-o", str(lib)],
                   check=True)
    L = C.CDLL(str(lib))
    for name in ("zd_solo", "zd_team"):
        f = getattr(L, name)
        f.restype = C.c_longlong
        f.argtypes = [C.c_void_p, C.c_ulonglong, C.c_void_p, C.c_ulonglong]
    return L


def _zstd():
    from xnyzip_b200 import _native as N
    z = C.CDLL(N.default_zstd_library())
    z.ZSTD_compressBound.restype = C.c_size_t
    z.ZSTD_compressBound.argtypes = [C.c_size_t]
    z.ZSTD_compress.restype = C.c_size_t
    z.ZSTD_compress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int]

    def frame(b, level):
        cap = z.ZSTD_compressBound(len(b))
        out = C.create_string_buffer(cap)
        size = z.ZSTD_compress(out, cap, b, len(b), level)
        return out.raw[:size]
    return frame


def _data():
    rng = np.random.default_rng(7)
    parts = []
    for _ in range(24):
        k, n = int(rng.integers(0, 4)), int(rng.integers(1, 20000))
        parts.append(rng.integers(0, 256, n, dtype=np.uint8).tobytes() if k == 0 else
                     bytes([int(rng.integers(0, 256))]) * n if k == 1 else
                     rng.geometric(float(rng.uniform(0.05, 0.9)), n).astype(np.uint8).tobytes() if k == 2 else
                     parts[int(rng.integers(0, len(parts)))][:n] if parts else b"abc")
    return [b"", b"q", b"The quick brown fox jumps over the lazy dog. " * 4000,
            rng.geometric(0.3, 200000).astype(np.uint8).tobytes(), bytes(150000), b"".join(parts)]


@pytest.mark.parametrize("team", ["zd_solo", "zd_team"])
def test_host_decoder_matches_libzstd(zd, team):
    frame = _zstd()
    fn = getattr(zd, team)
    for level in (1, 3, 19):
        for d in _data():
            f = frame(d, level)
            out = C.create_string_buffer(len(d) + 1)
            assert fn(f, len(f), out, len(d)) == len(d)
            assert out.raw[:len(d)] == d


ASAN_MAIN = r"""
#include "zstd_dec.cuh"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
int main(int argc, char** argv) {
    FILE* f = std::fopen(argv[1], "rb");
    std::vector<unsigned char> s(1 << 16);
    const size_t n = std::fread(s.data(), 1, s.size(), f);
    std::fclose(f);
    auto* ws = static_cast<xnyz::zd::Workspace*>(std::malloc(sizeof(xnyz::zd::Workspace)));
    std::vector<unsigned char> d(4096);
    const long long r = xnyz::zd::decode_frame(s.data(), n, d.data(), d.size(), *ws, xnyz::zd::SoloTeam{});
    std::free(ws);
    std::printf("%lld\n", r);
    return 0;
}
"""


def test_host_decoder_256_huffman_weights(tmp_path):
    """A Huffman tree description whose FSE-coded weights run to 256 entries is refused with a
    negative code, and (under AddressSanitizer) the decoder writes nothing past its weight
    array; libzstd refuses the same frame."""
    from zstd_craft import frame_with_huf_tree, huf_tree_256_weights
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    shutil.copy(HEADER, tmp_path / "zstd_dec.cuh")
    (tmp_path / "m.cpp").write_text(ASAN_MAIN)
    exe = tmp_path / "zd_asan"
    subprocess.run([cxx, "-O1", "-g", "-std=c++20", "-fsanitize=address,undefined", "-fno-sanitize-recover=all",
                    str(tmp_path / "m.cpp"), "-o", str(exe)], check=True)
    frame = frame_with_huf_tree(huf_tree_256_weights())
    (tmp_path / "f.bin").write_bytes(frame)
    r = subprocess.run([str(exe), str(tmp_path / "f.bin")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
    assert int(r.stdout.strip()) < 0
    z = C.CDLL(__import__("xnyzip_b200._native", fromlist=["x"]).default_zstd_library())
    z.ZSTD_decompress.restype = C.c_size_t
    z.ZSTD_decompress.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t]
    z.ZSTD_isError.restype = C.c_uint
    z.ZSTD_isError.argtypes = [C.c_size_t]
    out = C.create_string_buffer(256)
    assert z.ZSTD_isError(z.ZSTD_decompress(out, 256, frame, len(frame)))


@pytest.mark.parametrize("team", ["zd_solo", "zd_team"])
def test_host_decoder_damaged_frames(zd, team):
    frame = _zstd()
    fn = getattr(zd, team)
    d = _data()[-1]
    f = frame(d, 3)
    rng = np.random.default_rng(3)
    out = C.create_string_buffer(len(d) + 64)
    assert fn(f[:len(f) // 2], len(f) // 2, out, len(d)) < 0
    assert fn(f, len(f), out, len(d) - 1) < 0
    for _ in range(40):  # bit flips and overwritten tails: any status, never a disagreement
        g = bytearray(f)
        if rng.integers(0, 2):
            i = int(rng.integers(0, len(g)))
            g[i] ^= 1 << int(rng.integers(0, 8))
        else:
            i = int(rng.integers(4, len(g)))
            g[i:] = rng.integers(0, 256, len(g) - i, dtype=np.uint8).tobytes()
        assert fn(bytes(g), len(g), out, len(d) + 64) != -100
