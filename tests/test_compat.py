"""The C++ drop-in header include/xnyz_compat.hpp (the reference's composer class names over
the C ABI): it compiles against an Eigen-like point type and without Eigen, and on the GPU a
program written against the reference's classes produces the reference's frames and points
(byte for byte), its profile frames and cell tables, and its exception types."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")
SHIM = os.path.join(ROOT, "oracle", "shim")  # a minimal Eigen stand-in (test infrastructure)
LIBDIR = os.path.join(ROOT, "xnyzip_b200")

# A reference-style caller: only XnYZip:: names and Eigen types.  Reads n points, writes, for
# each mode, the frame and the decoded points; then the shared-codebook and cell-table calls
# and the exception paths.
PROGRAM = r"""
#include "xnyz_compat.hpp"
#include <cstdio>
#include <fstream>
#include <iterator>
#include <string>
using namespace XnYZip;
using P = Vec3<float>;

static void put(const std::string& path, const void* p, size_t n) {
    std::ofstream o(path, std::ios::binary);
    o.write(static_cast<const char*>(p), static_cast<std::streamsize>(n));
}
template <class V> static void put_pts(const std::string& path, const V& v) { put(path, v.data(), v.size() * 12); }

int main(int argc, char** argv) {
    std::ifstream f(argv[1], std::ios::binary);
    std::vector<char> raw((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    const std::string out = argv[2];
    std::vector<P> pts(raw.size() / 12);
    for (size_t i = 0; i < pts.size(); ++i) {
        float v[3];
        std::memcpy(v, raw.data() + 12 * i, 12);
        pts[i] = P(v[0], v[1], v[2]);
    }
    const QUANTIZER_TYPE qs[2] = {QUANTIZER_TYPE::CUBE, QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON};
    for (int q = 0; q < 2; ++q)
        for (int hil = 0; hil < 2; ++hil) {
            const std::string tag = std::to_string(q) + "_" + std::to_string(hil);
            auto a = pts;
            auto fr = BlockCompressor<float>(qs[q], 0.05f).compress(a, hil != 0);
            put(out + "/normal_" + tag + ".frame", fr.data(), fr.size());
            put_pts(out + "/normal_" + tag + ".sorted", a);
            put_pts(out + "/normal_" + tag + ".points", BlockDecompressor<float>(qs[q], 0.05f).decompress(fr));
            auto b = pts;
            auto fr2 = BlockCompressorRLE<float>(qs[q], 0.05f).compress(b, hil != 0);
            put(out + "/rle_" + tag + ".frame", fr2.data(), fr2.size());
            put_pts(out + "/rle_" + tag + ".points", BlockDecompressorRLE<float>(qs[q], 0.05f).decompress(fr2));
        }
    {   // shared codebooks: fit on the first half, code the second half with that profile
        std::vector<P> a(pts.begin(), pts.begin() + pts.size() / 2), b(pts.begin() + pts.size() / 2, pts.end());
        BlockCompressor<float> c(QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON, 0.05f);
        auto [fa, prof] = c.fit_profile(a, true);
        auto fb = c.compress_with_profile(b, true, prof);
        put(out + "/profile_fit.frame", fa.data(), fa.size());
        const auto blob = serialize_profile(prof);
        put(out + "/profile.bin", blob.data(), blob.size());
        put(out + "/profile_with.frame", fb.data(), fb.size());
        try {
            c.compress_with_profile(b, true, BlockEncodingProfile{});
            return 3;
        } catch (const std::runtime_error&) {
        }
    }
    {   // cell tables of a -rle frame, expanded back to points
        auto a = pts;
        auto fr = BlockCompressorRLE<float>(QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON, 0.05f).compress(a, true);
        BlockDecompressorRLE<float> d(QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON, 0.05f);
        auto t = d.decompress_to_cells(fr);
        put(out + "/cells.bin", t.cells.data(), t.cells.size() * 12);
        put(out + "/counts.bin", t.counts.data(), t.counts.size() * 4);
        put_pts(out + "/expanded.points", d.expand_cells_to_points(t));
        auto re = BlockCompressorRLE<float>(QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON, 0.05f)
                      .encode_cells_with_counts(t.cells, t.counts, t.range_x, t.range_y, t.range_z, t.offset, true);
        put(out + "/cells_reencoded.frame", re.data(), re.size());
    }
    try {  // damaged frame: the reference throws std::runtime_error
        std::vector<uint8_t> junk(64, 0x5A);
        BlockDecompressor<float>(QUANTIZER_TYPE::CUBE, 0.05f).decompress(junk);
        return 4;
    } catch (const std::runtime_error&) {
    }
    std::printf("ok\n");
    return 0;
}
"""


def _compile(tmp_path, eigen: bool):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libxnyz.so")):
        pytest.skip("libxnyz.so is not built")
    src = tmp_path / "compat_main.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / ("compat_eigen" if eigen else "compat_plain")
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", INCLUDE, str(src), "-o", str(exe), "-L", LIBDIR,
           "-lxnyz", f"-Wl,-rpath,{LIBDIR}"]
    cmd[3:3] = ["-I", SHIM] if eigen else ["-DXNYZ_COMPAT_NO_EIGEN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


@pytest.mark.parametrize("eigen", [True, False])
def test_compat_header_compiles(tmp_path, eigen):
    _compile(tmp_path, eigen)


@pytest.mark.gpu
@pytest.mark.parametrize("eigen", [True, False])
def test_compat_classes_match_reference(tmp_path, reference, eigen):
    from conftest import quiet_call
    from xnyzip_b200 import synthetic as S
    exe = _compile(tmp_path, eigen)
    x = S.terrain(30_000, 41, extent=400.0, amplitude=3.0, wavelength=150.0)
    x.tofile(tmp_path / "in.bin")
    out = tmp_path / "out"
    out.mkdir()
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])

    def rd(name, dtype=np.uint8):
        return np.fromfile(out / name, dtype=dtype)

    for q, qn in ((0, "cube"), (1, "to")):
        for hil in (0, 1):
            tag = f"{q}_{hil}"
            fr, srt = quiet_call(reference, reference.compress, x, qn, 0.05, hil, 0, with_sorted=True)
            assert rd(f"normal_{tag}.frame").tobytes() == fr
            want = quiet_call(reference, reference.decompress, fr, qn, 0.05, 0)
            assert rd(f"normal_{tag}.points", np.float32).tobytes() == want.tobytes()
            # compress() reorders its argument into container order; points of one lattice cell
            # may come in another order than libstdc++'s introsort leaves them
            got = rd(f"normal_{tag}.sorted", np.float32).reshape(-1, 3)
            diff = np.flatnonzero((got != srt).any(axis=1))
            assert np.array_equal(np.sort(got.view("V12").ravel()), np.sort(srt.view("V12").ravel()))
            for i in diff:  # a differing position lies in a run of one cell: its decoded neighbour agrees
                assert (want[i] == want[max(i - 1, 0)]).all() or (want[i] == want[min(i + 1, len(want) - 1)]).all()
            fr = quiet_call(reference, reference.compress, x, qn, 0.05, hil, 1)
            assert rd(f"rle_{tag}.frame").tobytes() == fr
            want = quiet_call(reference, reference.decompress, fr, qn, 0.05, 1)
            assert rd(f"rle_{tag}.points", np.float32).tobytes() == want.tobytes()
    half = x.shape[0] // 2
    fa, prof = quiet_call(reference, reference.fit_profile, x[:half], "to", 0.05, 1)
    assert rd("profile_fit.frame").tobytes() == fa
    assert rd("profile.bin").tobytes() == prof
    fb = quiet_call(reference, reference.compress_with_profile, x[half:], "to", 0.05, 1, prof)
    assert rd("profile_with.frame").tobytes() == fb
    fr = quiet_call(reference, reference.compress, x, "to", 0.05, 1, 1)
    cells, counts, off, rng, hil = quiet_call(reference, reference.decompress_to_cells, fr)
    assert rd("cells.bin", np.int32).tobytes() == cells.tobytes()
    assert rd("counts.bin", np.int32).tobytes() == counts.tobytes()
    want = quiet_call(reference, reference.expand_cells, cells, counts, off)
    assert rd("expanded.points", np.float32).tobytes() == want.tobytes()
    re = quiet_call(reference, reference.encode_cells, cells, counts, rng, off, hil)
    assert rd("cells_reencoded.frame").tobytes() == re
