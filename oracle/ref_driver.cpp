// Thin extern "C" driver around the UNMODIFIED XnYZip reference headers.
//
// Test infrastructure only.  Built by oracle/build_ref.sh from the reference sources where
// they lie (include path = the reference's source/ directory) into oracle/_ref/, together
// with the project's Eigen/zstd declaration shims under oracle/shim/.  Nothing here is
// part of the product; tests, smoke() and bench.py's CPU baseline are its only callers.
//
// Each entry point calls the reference's own classes and functions; the composer-level
// entry points run exactly BlockCompressor{,RLE}<float>::compress and
// BlockDecompressor{,RLE}<float>::decompress (composer/block_compressor.hpp:39,
// composer/block_compressor_rle.hpp:38, composer/block_decompressor.hpp:31,
// composer/block_decompressor_rle.hpp:32).
#include "lib.hpp"

#include <fcntl.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <vector>

namespace {

using P3 = Eigen::RowVector3f;

XnYZip::QUANTIZER_TYPE qtype(int q) {
    if (q == 2) return XnYZip::QUANTIZER_TYPE::ADAPTIVE;
    return q == 1 ? XnYZip::QUANTIZER_TYPE::TRUNCATED_OCTAHEDRON : XnYZip::QUANTIZER_TYPE::CUBE;
}

std::vector<P3> to_points(const float* xyz, uint64_t n) {
    std::vector<P3> pts;
    pts.reserve(n);
    for (uint64_t i = 0; i < n; ++i) pts.emplace_back(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return pts;
}

template <typename V>
uint8_t* dup_bytes(const V& v, uint64_t* len) {
    *len = v.size() * sizeof(typename V::value_type);
    uint8_t* p = static_cast<uint8_t*>(std::malloc(*len ? *len : 1));
    if (*len) std::memcpy(p, v.data(), *len);
    return p;
}

int g_saved_stdout = -1;

}  // namespace

extern "C" {

void ref_free(void* p) { std::free(p); }

// Redirect the process's stdout to /dev/null (the reference prints diagnostics on every
// call); ref_quiet(0) restores it.
void ref_quiet(int on) {
    std::cout.flush();
    std::fflush(stdout);
    if (on && g_saved_stdout < 0) {
        g_saved_stdout = dup(1);
        int fd = open("/dev/null", O_WRONLY);
        dup2(fd, 1);
        close(fd);
    } else if (!on && g_saved_stdout >= 0) {
        dup2(g_saved_stdout, 1);
        close(g_saved_stdout);
        g_saved_stdout = -1;
    }
}

// Full compressor: returns the zstd frame.  If sorted_xyz is non-null it receives the
// input points as compress() leaves them (it reorders its argument).
int ref_compress(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, int rle,
                 int direct_threshold, uint8_t** out, uint64_t* out_len, float* sorted_xyz) {
    try {
        auto pts = to_points(xyz, n);
        std::vector<uint8_t> bytes;
        if (rle) {
            XnYZip::BlockCompressorRLE<float> c(qtype(quantizer), l2, false, direct_threshold);
            bytes = c.compress(pts, hilbert != 0);
        } else {
            XnYZip::BlockCompressor<float> c(qtype(quantizer), l2, false, direct_threshold);
            bytes = c.compress(pts, hilbert != 0);
        }
        if (sorted_xyz)
            for (uint64_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) sorted_xyz[3 * i + k] = pts[i][k];
        *out = dup_bytes(bytes, out_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_compress: %s\n", e.what());
        return 1;
    }
}

// BlockCompressor::fit_profile: the zstd frame and serialize_profile of the profile.
int ref_fit_profile(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, int direct_threshold,
                    uint8_t** out, uint64_t* out_len, uint8_t** prof, uint64_t* prof_len, float* sorted_xyz) {
    try {
        auto pts = to_points(xyz, n);
        XnYZip::BlockCompressor<float> c(qtype(quantizer), l2, false, direct_threshold);
        auto [bytes, profile] = c.fit_profile(pts, hilbert != 0);
        const auto blob = XnYZip::serialize_profile(profile);
        if (sorted_xyz)
            for (uint64_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) sorted_xyz[3 * i + k] = pts[i][k];
        *out = dup_bytes(bytes, out_len);
        *prof = dup_bytes(blob, prof_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_fit_profile: %s\n", e.what());
        return 1;
    }
}

// BlockCompressor::compress_with_profile with deserialize_profile(blob).
int ref_compress_with_profile(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert,
                              int direct_threshold, const uint8_t* prof, uint64_t prof_len, uint8_t** out,
                              uint64_t* out_len) {
    try {
        auto pts = to_points(xyz, n);
        XnYZip::BlockCompressor<float> c(qtype(quantizer), l2, false, direct_threshold);
        const auto profile = XnYZip::deserialize_profile(std::vector<uint8_t>(prof, prof + prof_len));
        auto bytes = c.compress_with_profile(pts, hilbert != 0, profile);
        *out = dup_bytes(bytes, out_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_compress_with_profile: %s\n", e.what());
        return 1;
    }
}

int ref_decompress(const uint8_t* buf, uint64_t len, int quantizer, float l2, int rle, float** xyz_out,
                   uint64_t* n_out) {
    try {
        std::vector<uint8_t> bytes(buf, buf + len);
        std::vector<P3> pts;
        if (rle) {
            XnYZip::BlockDecompressorRLE<float> d(qtype(quantizer), l2);
            pts = d.decompress(bytes);
        } else {
            XnYZip::BlockDecompressor<float> d(qtype(quantizer), l2);
            pts = d.decompress(bytes);
        }
        *n_out = pts.size();
        float* o = static_cast<float*>(std::malloc(pts.size() * 12 + 4));
        for (size_t i = 0; i < pts.size(); ++i)
            for (int k = 0; k < 3; ++k) o[3 * i + k] = pts[i][k];
        *xyz_out = o;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_decompress: %s\n", e.what());
        return 1;
    }
}

// zstd frame -> pre-zstd container bytes (composer/utils.hpp:11).
int ref_unzstd(const uint8_t* buf, uint64_t len, uint8_t** out, uint64_t* out_len) {
    try {
        std::vector<uint8_t> bytes(buf, buf + len);
        auto raw = XnYZip::decompress_buffer(bytes);
        *out = dup_bytes(raw, out_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_unzstd: %s\n", e.what());
        return 1;
    }
}

// Compress then decompress, each timed with the reference's own Timer
// (statistics/timer.hpp) exactly as source/main.cpp:85-100 does.
int ref_roundtrip_timed(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, int rle,
                        int direct_threshold, double* t_compress, double* t_decompress, uint64_t* comp_bytes,
                        uint64_t* n_decoded) {
    try {
        auto pts = to_points(xyz, n);
        XnYZip::Timer timer;
        std::vector<uint8_t> bytes;
        std::vector<P3> rec;
        if (rle) {
            timer.start();
            XnYZip::BlockCompressorRLE<float> c(qtype(quantizer), l2, false, direct_threshold);
            bytes = c.compress(pts, hilbert != 0);
            *t_compress = timer.stop();
            timer.start();
            XnYZip::BlockDecompressorRLE<float> d(qtype(quantizer), l2);
            rec = d.decompress(bytes);
            *t_decompress = timer.stop();
        } else {
            timer.start();
            XnYZip::BlockCompressor<float> c(qtype(quantizer), l2, false, direct_threshold);
            bytes = c.compress(pts, hilbert != 0);
            *t_compress = timer.stop();
            timer.start();
            XnYZip::BlockDecompressor<float> d(qtype(quantizer), l2);
            rec = d.decompress(bytes);
            *t_decompress = timer.stop();
        }
        *comp_bytes = bytes.size();
        *n_decoded = rec.size();
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_roundtrip_timed: %s\n", e.what());
        return 1;
    }
}

// ---- stage-level entry points --------------------------------------------------------

// shift_points + quantize (preprocessor/shifting.hpp:11, *_quantizer.hpp::quantize).
int ref_quantize(const float* xyz, uint64_t n, int quantizer, float l2, float* offset3, int32_t* q_out) {
    auto pts = to_points(xyz, n);
    Eigen::RowVector3f offset;
    auto shifted = XnYZip::shift_points<float>(pts, offset);
    std::unique_ptr<XnYZip::BaseQuantizer<float>> qz;
    if (quantizer == 1)
        qz = std::make_unique<XnYZip::TruncatedOctahedronQuantizer<float>>(l2);
    else
        qz = std::make_unique<XnYZip::CubeQuantizer<float>>(l2);
    std::vector<float> params;
    auto q = qz->quantize(shifted, params);
    for (int k = 0; k < 3; ++k) offset3[k] = offset[k];
    for (uint64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) q_out[3 * i + k] = q[i][k];
    return 0;
}

// quantizer->recover + unshift_points.
int ref_recover(const int32_t* q, uint64_t n, int quantizer, float l2, const float* offset3, float* xyz_out) {
    std::vector<Eigen::RowVector3i> cells;
    cells.reserve(n);
    for (uint64_t i = 0; i < n; ++i) cells.emplace_back(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    std::unique_ptr<XnYZip::BaseQuantizer<float>> qz;
    if (quantizer == 1)
        qz = std::make_unique<XnYZip::TruncatedOctahedronQuantizer<float>>(l2);
    else
        qz = std::make_unique<XnYZip::CubeQuantizer<float>>(l2);
    std::vector<float> params;
    auto rec = qz->recover(cells, params);
    auto un = XnYZip::unshift_points(rec, Eigen::RowVector3f(offset3[0], offset3[1], offset3[2]));
    for (uint64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) xyz_out[3 * i + k] = un[i][k];
    return 0;
}

uint64_t ref_morton(int x, int y, int z) { return XnYZip::morton_code(Eigen::RowVector3i(x, y, z)); }
void ref_m2h(const uint64_t* in, uint64_t n, unsigned iter, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = mve::mortonToHilbert3(in[i], iter);
}
void ref_h2m(const uint64_t* in, uint64_t n, unsigned iter, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = mve::hilbertToMorton3(in[i], iter);
}

struct RefLCP {
    uint64_t nblocks, n;
    uint64_t* blkst;
    uint64_t* blkcnt;
    uint8_t* quads;
    uint64_t* repos;
    uint64_t* ords;
};

// block_quantize (quantizer/block_quantizer.hpp:84) on lattice cells with 64^3 sub-blocks.
int ref_block_quantize(const int32_t* q, uint64_t n, int rx, int ry, int rz, int hilbert, RefLCP* out) {
    std::vector<Eigen::RowVector3i> cells;
    cells.reserve(n);
    for (uint64_t i = 0; i < n; ++i) cells.emplace_back(q[3 * i], q[3 * i + 1], q[3 * i + 2]);
    auto m = block_quantize(cells, 64, 64, 64, rx, ry, rz, hilbert != 0);
    uint64_t l;
    out->nblocks = m.blkst.size();
    out->n = m.repos.size();
    out->blkst = reinterpret_cast<uint64_t*>(dup_bytes(m.blkst, &l));
    out->blkcnt = reinterpret_cast<uint64_t*>(dup_bytes(m.blkcnt, &l));
    out->quads = dup_bytes(m.quads, &l);
    out->repos = reinterpret_cast<uint64_t*>(dup_bytes(m.repos, &l));
    std::vector<uint64_t> ords(m.ords.begin(), m.ords.end());
    out->ords = reinterpret_cast<uint64_t*>(dup_bytes(ords, &l));
    return 0;
}

// recover_from_lcp_meta (quantizer/block_quantizer.hpp:154) -> int cells.
int ref_recover_lcp(const uint64_t* blkst, const uint64_t* blkcnt, uint64_t nblocks, const uint8_t* quads,
                    const uint64_t* repos, uint64_t n, int rx, int ry, int rz, int hilbert, int32_t* cells_out) {
    LCPMeta m;
    m.blkst.assign(blkst, blkst + nblocks);
    m.blkcnt.assign(blkcnt, blkcnt + nblocks);
    m.quads.assign(quads, quads + n);
    m.repos.assign(repos, repos + n);
    m.is_hilbert = hilbert != 0;
    auto c = recover_from_lcp_meta<int>(m, 64, 64, 64, rx, ry, rz);
    for (size_t i = 0; i < c.size(); ++i)
        for (int k = 0; k < 3; ++k) cells_out[3 * i + k] = c[i][k];
    return 0;
}

// HuffmanEncoder<T> build/get_meta/encode (encoder/huffman_encoder.hpp:33,126,150).
// kind: 0 = uint64_t, 1 = uint8_t, 2 = int.
int ref_huffman(int kind, const void* data, uint64_t n, int force_exp_golomb, uint8_t** meta, uint64_t* meta_len,
                uint8_t** enc, uint64_t* enc_len) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        const T* d = static_cast<const T*>(data);
        std::vector<T> v(d, d + n);
        XnYZip::HuffmanEncoder<T> h;
        if (force_exp_golomb) h.set_use_exp_golomb(true);
        h.build(v);
        auto m = h.get_meta();
        auto e = h.encode(v);
        *meta = dup_bytes(m, meta_len);
        *enc = dup_bytes(e, enc_len);
    };
    if (kind == 0) run(uint64_t{});
    else if (kind == 1) run(uint8_t{});
    else run(int{});
    return 0;
}

int ref_huffman_decode(int kind, const uint8_t* meta, uint64_t meta_len, const uint8_t* enc, uint64_t enc_len,
                       uint64_t n, void* out, uint64_t* n_out) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        XnYZip::HuffmanEncoder<T> h;
        h.load_meta(std::vector<uint8_t>(meta, meta + meta_len));
        auto v = h.decode(std::vector<uint8_t>(enc, enc + enc_len), n);
        *n_out = v.size();
        std::memcpy(out, v.data(), v.size() * sizeof(T));
    };
    if (kind == 0) run(uint64_t{});
    else if (kind == 1) run(uint8_t{});
    else run(int{});
    return 0;
}

// GolombRiceCoder<T>::pack / BitPacker<uint64_t>::pack.  kind 0 = uint64_t, 1 = uint8_t.
int ref_gr_pack(int kind, const void* data, uint64_t n, uint8_t** meta, uint64_t* meta_len, uint8_t** enc,
                uint64_t* enc_len) {
    BitpackResult r;
    if (kind == 0) {
        const uint64_t* d = static_cast<const uint64_t*>(data);
        r = GolombRiceCoder<uint64_t>::pack(std::vector<uint64_t>(d, d + n));
    } else {
        const uint8_t* d = static_cast<const uint8_t*>(data);
        r = GolombRiceCoder<uint8_t>::pack(std::vector<uint8_t>(d, d + n));
    }
    *meta = dup_bytes(r.meta, meta_len);
    *enc = dup_bytes(r.data, enc_len);
    return 0;
}

int ref_bitpack(const uint64_t* data, uint64_t n, uint8_t** meta, uint64_t* meta_len, uint8_t** enc,
                uint64_t* enc_len) {
    try {
        auto r = BitPacker<uint64_t>::pack(std::vector<uint64_t>(data, data + n));
        *meta = dup_bytes(r.meta, meta_len);
        *enc = dup_bytes(r.data, enc_len);
        return 0;
    } catch (const std::exception& e) {
        return 1;
    }
}

// Distributed-RLE cell API (composer/block_compressor_rle.hpp:341-470,
// composer/block_decompressor_rle.hpp:230-358): cells are int32 xyz triples.
int ref_encode_cells(const int32_t* cells, const int32_t* counts, uint64_t n, int rx, int ry, int rz,
                     const float* offset3, int hilbert, int quantizer, float l2, uint8_t** out, uint64_t* out_len) {
    try {
        std::vector<Eigen::RowVector3i> c;
        c.reserve(n);
        for (uint64_t i = 0; i < n; ++i) c.emplace_back(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2]);
        std::vector<int> k(counts, counts + n);
        XnYZip::BlockCompressorRLE<float> enc(qtype(quantizer), l2);
        auto bytes = enc.encode_cells_with_counts(c, k, rx, ry, rz, P3(offset3[0], offset3[1], offset3[2]), hilbert != 0);
        *out = dup_bytes(bytes, out_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_encode_cells: %s\n", e.what());
        return 1;
    }
}

int ref_decompress_to_cells(const uint8_t* buf, uint64_t len, int quantizer, float l2, int32_t** cells_out,
                            int32_t** counts_out, uint64_t* n_out, float* offset3, int32_t* ranges3, int* hilbert) {
    try {
        std::vector<uint8_t> bytes(buf, buf + len);
        XnYZip::BlockDecompressorRLE<float> d(qtype(quantizer), l2);
        auto t = d.decompress_to_cells(bytes);
        *n_out = t.cells.size();
        int32_t* c = static_cast<int32_t*>(std::malloc(t.cells.size() * 12 + 4));
        int32_t* k = static_cast<int32_t*>(std::malloc(t.counts.size() * 4 + 4));
        for (size_t i = 0; i < t.cells.size(); ++i)
            for (int a = 0; a < 3; ++a) c[3 * i + a] = t.cells[i][a];
        for (size_t i = 0; i < t.counts.size(); ++i) k[i] = t.counts[i];
        *cells_out = c;
        *counts_out = k;
        for (int a = 0; a < 3; ++a) offset3[a] = t.offset[a];
        ranges3[0] = t.range_x;
        ranges3[1] = t.range_y;
        ranges3[2] = t.range_z;
        *hilbert = t.is_hilbert;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_decompress_to_cells: %s\n", e.what());
        return 1;
    }
}

int ref_expand_cells(const int32_t* cells, const int32_t* counts, uint64_t n, const float* offset3, int quantizer,
                     float l2, float** xyz_out, uint64_t* n_out) {
    try {
        XnYZip::BlockDecompressorRLE<float> d(qtype(quantizer), l2);
        XnYZip::BlockDecompressorRLE<float>::DecodedCellTable t;
        for (uint64_t i = 0; i < n; ++i) {
            t.cells.emplace_back(cells[3 * i], cells[3 * i + 1], cells[3 * i + 2]);
            t.counts.push_back(counts[i]);
        }
        t.offset = P3(offset3[0], offset3[1], offset3[2]);
        auto pts = d.expand_cells_to_points(t);
        *n_out = pts.size();
        float* o = static_cast<float*>(std::malloc(pts.size() * 12 + 4));
        for (size_t i = 0; i < pts.size(); ++i)
            for (int a = 0; a < 3; ++a) o[3 * i + a] = pts[i][a];
        *xyz_out = o;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_expand_cells: %s\n", e.what());
        return 1;
    }
}

}  // extern "C"
