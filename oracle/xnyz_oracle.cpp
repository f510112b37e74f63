// ORACLE — test infrastructure only.  A sequential CPU restatement of the XnYZip
// compress/decompress path, written for this project and used solely as the checker by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  The product never links,
// imports or calls it.
//
// Parity pin: tests/test_oracle_vs_ref.py compares every function here with the reference
// itself (compiled from its own sources into oracle/_ref by oracle/build_ref.sh) and with
// the committed fixtures under tests/golden/ that were generated from it.
//
// Every function cites the reference file:line (paths relative to the reference's
// source/ directory) whose behaviour it restates.  Container layout: composer/
// block_compressor.hpp:56-215 and block_compressor_rle.hpp:91-314.
//
// The Huffman stage deliberately uses std::unordered_map / std::priority_queue exactly as
// the reference does (encoder/huffman_encoder.hpp:43-123): their iteration and
// tie-breaking order is part of the stream format.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <queue>
#include <set>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include <dlfcn.h>

namespace {

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;
using i32 = int32_t;
using Bytes = std::vector<u8>;

// ---------------------------------------------------------------- zstd (runtime) ----
struct Zstd {
    size_t (*compressBound)(size_t) = nullptr;
    size_t (*compress)(void*, size_t, const void*, size_t, int) = nullptr;
    size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
    unsigned long long (*frameContentSize)(const void*, size_t) = nullptr;
    unsigned (*isError)(size_t) = nullptr;
    bool ok = false;
};
Zstd g_zstd;
char g_zstd_path[4096] = {0};

bool zstd_load() {
    if (g_zstd.ok) return true;
    const char* path = g_zstd_path[0] ? g_zstd_path : getenv("XNYZ_ZSTD_LIBRARY");
    if (!path) return false;
    void* h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return false;
    g_zstd.compressBound = (size_t(*)(size_t))dlsym(h, "ZSTD_compressBound");
    g_zstd.compress = (size_t(*)(void*, size_t, const void*, size_t, int))dlsym(h, "ZSTD_compress");
    g_zstd.decompress = (size_t(*)(void*, size_t, const void*, size_t))dlsym(h, "ZSTD_decompress");
    g_zstd.frameContentSize = (unsigned long long (*)(const void*, size_t))dlsym(h, "ZSTD_getFrameContentSize");
    g_zstd.isError = (unsigned (*)(size_t))dlsym(h, "ZSTD_isError");
    g_zstd.ok = g_zstd.compressBound && g_zstd.compress && g_zstd.decompress && g_zstd.frameContentSize &&
                g_zstd.isError;
    return g_zstd.ok;
}

// ---------------------------------------------------------- float -> int (x86) ------
// static_cast<int>(float) as gcc compiles it on x86-64 (cvttss2si): truncation, and
// 0x80000000 for NaN or out-of-range values.
inline i32 f2i(float f) {
    if (!(f > -2147483904.0f && f < 2147483648.0f)) return INT32_MIN;
    return static_cast<i32>(f);
}

// ------------------------------------------------------------------ quantizers ------
// TruncatedOctahedronQuantizer::quantize (quantizer/truncated_octahedron_quantizer.hpp:21-55)
// with Eigen's coefficient-wise semantics; squaredNorm is c0 + (c1 + c2) (Eigen 3.4.0's
// unrolled reduction order).
struct QConst {
    float div;     // quantize divisor: float(double(2*s) / sqrt(k))
    float s;       // the L2 bound as float
    float rsqrt;   // recover divisor float(sqrt(k))
};

QConst make_const(int quantizer, float l2) {
    double k = quantizer == 1 ? 5.0 : 3.0;
    QConst c;
    c.s = l2;
    c.div = static_cast<float>(static_cast<double>(2.0f * l2) / std::sqrt(k));
    c.rsqrt = static_cast<float>(std::sqrt(k));
    return c;
}

void quantize_to(const float p[3], float div, i32 out[3]) {
    float q[3], e[3], o[3];
    for (int k = 0; k < 3; ++k) q[k] = p[k] / div;
    for (int k = 0; k < 3; ++k) {
        e[k] = std::round(q[k] * 0.5f) * 2.0f;
        o[k] = std::round((q[k] - 1.0f) * 0.5f) * 2.0f + 1.0f;
    }
    float de0 = (q[0] - e[0]) * (q[0] - e[0]), de1 = (q[1] - e[1]) * (q[1] - e[1]), de2 = (q[2] - e[2]) * (q[2] - e[2]);
    float do0 = (q[0] - o[0]) * (q[0] - o[0]), do1 = (q[1] - o[1]) * (q[1] - o[1]), do2 = (q[2] - o[2]) * (q[2] - o[2]);
    float dE = de0 + (de1 + de2);
    float dO = do0 + (do1 + do2);
    const float* pick = (dE <= dO) ? e : o;
    i32 n[3] = {f2i(pick[0]), f2i(pick[1]), f2i(pick[2])};
    if (n[0] & 1) {
        n[0] = (n[0] + 1) >> 1;
        n[1] = (n[1] + 1) >> 1;
    } else {
        n[0] >>= 1;
        n[1] >>= 1;
    }
    out[0] = n[0];
    out[1] = n[1];
    out[2] = n[2];
}

// CubeQuantizer::quantize (quantizer/cube_quantizer.hpp:15-27).
void quantize_cube(const float p[3], float div, i32 out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = f2i(std::floor(p[k] / div));
}

// TruncatedOctahedronQuantizer::recover (:57-76): ((v * 2) * s) / float(sqrt 5).
void recover_to(const i32 c[3], const QConst& k, float out[3]) {
    i32 n[3] = {c[0], c[1], c[2]};
    if (n[2] & 1) {
        n[0] = static_cast<i32>(static_cast<u32>(n[0]) << 1) - 1;
        n[1] = static_cast<i32>(static_cast<u32>(n[1]) << 1) - 1;
    } else {
        n[0] = static_cast<i32>(static_cast<u32>(n[0]) << 1);
        n[1] = static_cast<i32>(static_cast<u32>(n[1]) << 1);
    }
    for (int d = 0; d < 3; ++d) out[d] = ((static_cast<float>(n[d]) * 2.0f) * k.s) / k.rsqrt;
}

// CubeQuantizer::recover (:29-38): (((v + 0.5) * 2) * s) / float(sqrt 3).
void recover_cube(const i32 c[3], const QConst& k, float out[3]) {
    for (int d = 0; d < 3; ++d) out[d] = (((static_cast<float>(c[d]) + 0.5f) * 2.0f) * k.s) / k.rsqrt;
}

// AdaptiveQuantizer (quantizer/adaptive_quantizer.hpp:16-97): per-axis steps from the
// extent of the shifted points, a = R * (max_x - min_x) / norm with norm the extent's
// length (R / sqrt(3) on every axis when norm is 0); the maxima start at the smallest
// normal float and the minima at FLT_MAX, as there.  Cells are round(p / step) cast to int,
// points idx * step.
void adaptive_steps(const float* xyz, u64 n, const float off[3], float R, float step[3]) {
    float mn[3], mx[3];
    for (int k = 0; k < 3; ++k) {
        mn[k] = std::numeric_limits<float>::max();
        mx[k] = std::numeric_limits<float>::min();
    }
    for (u64 i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            const float p = xyz[3 * i + k] - off[k];
            mn[k] = std::min(mn[k], p);
            mx[k] = std::max(mx[k], p);
        }
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    const float norm = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (norm > 0) {
        step[0] = R * dx / norm;
        step[1] = R * dy / norm;
        step[2] = R * dz / norm;
    } else {
        step[0] = step[1] = step[2] = R / std::sqrt(3.0f);
    }
}

void quantize_adaptive(const float p[3], const float step[3], i32 out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = f2i(std::round(p[k] / step[k]));
}

void recover_adaptive(const i32 c[3], const float step[3], float out[3]) {
    for (int k = 0; k < 3; ++k) out[k] = static_cast<float>(c[k]) * step[k];
}

// ------------------------------------------------------------------ Morton ------------
// split_by_3 / morton_code / compact_by_3 (preprocessor/z_order_curve.hpp:14-47):
// 21 bits per axis, x at bit 0, y at bit 1, z at bit 2.
u64 spread3(u32 v) {
    u64 x = v & 0x1fffffu, r = 0;
    for (int b = 0; b < 21; ++b) r |= ((x >> b) & 1ull) << (3 * b);
    return r;
}
u32 gather3(u64 m) {
    u32 r = 0;
    for (int b = 0; b < 21; ++b) r |= static_cast<u32>((m >> (3 * b)) & 1ull) << b;
    return r;
}
u64 morton(i32 x, i32 y, i32 z) {
    return spread3(static_cast<u32>(x)) | (spread3(static_cast<u32>(y)) << 1) | (spread3(static_cast<u32>(z)) << 2);
}

// ------------------------------------------------------------------ Hilbert -----------
// The digit-permutation Hilbert transform of quantizer/hilbert-curves-cpp/hilbert.cpp.
// Tables are rebuilt here from the same construction (:33-357): the 24 cube-rotation
// permutations in lexicographic order, then a depth-first search for each child's
// orientation so that consecutive children touch.
using Perm = std::array<u8, 8>;
constexpr Perm kH2M = {0, 1, 3, 2, 6, 7, 5, 4};  // base Gray-code pattern (:33,44)

Perm invert(const Perm& p) {
    Perm r{};
    for (int i = 0; i < 8; ++i) r[p[i]] = static_cast<u8>(i);
    return r;
}

struct HilbertTables {
    Perm m2h;              // mortonToHilbertPerm
    Perm childH2M[8];      // hilbertToMortonPermutations
    Perm childM2H[8];      // mortonToHilbertPermutations
};

std::array<int, 3> corner(int v) { return {(v >> 2) & 1, (v >> 1) & 1, v & 1}; }

bool hilbert_search(const std::vector<Perm>& rots, Perm out[8], int i, std::array<int, 3> prev_end) {
    auto pos = [](int child) { return corner(kH2M[child]); };
    std::array<int, 3> begin_g, end_g, cur_g;
    for (int k = 0; k < 3; ++k) {
        begin_g[k] = pos(0)[k] * 3;
        end_g[k] = pos(7)[k] * 3;
        cur_g[k] = pos(i)[k] * 2;
    }
    for (const Perm& r : rots) {
        auto b = corner(r[kH2M[0]]);
        std::array<int, 3> bg{b[0] + cur_g[0], b[1] + cur_g[1], b[2] + cur_g[2]};
        if (i == 0) {
            if (bg != begin_g) continue;
        } else {
            int d = 0;
            for (int k = 0; k < 3; ++k) d += (bg[k] - prev_end[k]) * (bg[k] - prev_end[k]);
            if (d != 1) continue;
        }
        auto e = corner(r[kH2M[7]]);
        std::array<int, 3> eg{e[0] + cur_g[0], e[1] + cur_g[1], e[2] + cur_g[2]};
        if (i != 7) {
            if (hilbert_search(rots, out, i + 1, eg)) {
                out[kH2M[i]] = r;
                return true;
            }
            continue;
        }
        if (eg != end_g) continue;
        out[kH2M[i]] = r;
        return true;
    }
    return false;
}

HilbertTables build_hilbert() {
    static const int sn[4] = {0, 1, 0, -1}, cs[4] = {1, 0, -1, 0};
    std::set<Perm> uniq;
    for (int rx = 0; rx < 4; ++rx)
        for (int ry = 0; ry < 4; ++ry)
            for (int rz = 0; rz < 4; ++rz) {
                int sx = sn[rx], sy = sn[ry], sz = sn[rz], cx = cs[rx], cy = cs[ry], cz = cs[rz];
                int m[3][3] = {{cx * cy, sx * sz - cx * cz * sy, cz * sx + cx * sy * sz},
                               {sy, cy * cz, -cy * sz},
                               {-cy * sx, cx * sz + cz * sx * sy, cx * cz - sx * sy * sz}};
                Perm p{};
                for (int i = 0; i < 8; ++i) {
                    int v[3] = {((i >> 2) & 1) * 2 - 1, ((i >> 1) & 1) * 2 - 1, (i & 1) * 2 - 1};
                    int r[3];
                    for (int k = 0; k < 3; ++k) r[k] = (m[k][0] * v[0] + m[k][1] * v[1] + m[k][2] * v[2] + 1) / 2;
                    p[i] = static_cast<u8>((r[0] << 2) | (r[1] << 1) | r[2]);
                }
                uniq.insert(p);
            }
    std::vector<Perm> rots(uniq.begin(), uniq.end());
    HilbertTables t{};
    t.m2h = invert(kH2M);
    hilbert_search(rots, t.childH2M, 0, {0, 0, 0});
    for (int i = 0; i < 8; ++i) t.childM2H[i] = invert(t.childH2M[i]);
    return t;
}

const HilbertTables& tables() {
    static const HilbertTables t = build_hilbert();
    return t;
}

inline u64 set_digit(u64 v, unsigned level, u64 d) {
    unsigned s = level * 3;
    return (v & ~(7ull << s)) | (d << s);
}

// mortonToHilbert3 (hilbert.cpp:439-464).
u64 m2h(u64 morton, unsigned iteration) {
    const auto& t = tables();
    u64 r = morton;
    for (unsigned i = iteration; i != 0; --i) {
        u8 md = (r >> (3 * i)) & 7;
        r = set_digit(r, i, t.m2h[md]);
        const Perm& p = t.childM2H[md];
        for (unsigned j = 0; j < i; ++j) r = set_digit(r, j, p[(r >> (3 * j)) & 7]);
    }
    return set_digit(r, 0, t.m2h[r & 7]);
}

// hilbertToMorton3 (hilbert.cpp:412-437).
u64 h2m(u64 hilbert, unsigned iteration) {
    const auto& t = tables();
    u64 r = set_digit(hilbert, 0, kH2M[hilbert & 7]);
    for (unsigned i = 1; i <= iteration; ++i) {
        u8 md = kH2M[(r >> (3 * i)) & 7];
        r = set_digit(r, i, md);
        const Perm& p = t.childH2M[md];
        for (unsigned j = 0; j < i; ++j) r = set_digit(r, j, p[(r >> (3 * j)) & 7]);
    }
    return r;
}

// ----------------------------------------------------------------- shift ------------
// shift_points (preprocessor/shifting.hpp:11-36): strict '<' scan from FLT_MAX.
void shift_offset(const float* xyz, u64 n, float off[3]) {
    off[0] = off[1] = off[2] = std::numeric_limits<float>::max();
    for (u64 i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k)
            if (xyz[3 * i + k] < off[k]) off[k] = xyz[3 * i + k];
}

// shift_points + quantize; `params` receives the quantizer's parameters (the adaptive
// steps; none for TO and cube).
void quantize_all(const float* xyz, u64 n, int quantizer, float l2, float off[3], std::vector<i32>& q,
                  std::vector<float>* params = nullptr) {
    shift_offset(xyz, n, off);
    QConst c = make_const(quantizer, l2);
    float step[3] = {0, 0, 0};
    if (quantizer == 2) adaptive_steps(xyz, n, off, l2, step);
    if (params) {
        params->clear();
        if (quantizer == 2) params->assign(step, step + 3);
    }
    q.resize(3 * n);
    for (u64 i = 0; i < n; ++i) {
        float p[3] = {xyz[3 * i] - off[0], xyz[3 * i + 1] - off[1], xyz[3 * i + 2] - off[2]};
        if (quantizer == 1)
            quantize_to(p, c.div, &q[3 * i]);
        else if (quantizer == 2)
            quantize_adaptive(p, step, &q[3 * i]);
        else
            quantize_cube(p, c.div, &q[3 * i]);
    }
}

// ------------------------------------------------------------- bit writers ----------
// BitPacker<uint64_t>::pack (encoder/bitpacking_encoder.hpp:17-51): width = bit length of
// the maximum (1 for all zeros), values LSB-first; meta = u32 n LE + u8 width.
void bitpack(const std::vector<u64>& v, Bytes& meta, Bytes& data) {
    if (v.empty()) throw std::invalid_argument("Input vector must not be empty");
    u64 mx = 0;
    for (u64 x : v) mx = std::max(mx, x);
    int w = mx == 0 ? 1 : 64 - __builtin_clzll(mx);
    u32 n = static_cast<u32>(v.size());
    meta = {u8(n), u8(n >> 8), u8(n >> 16), u8(n >> 24), u8(w)};
    data.assign((static_cast<u64>(n) * w + 7) / 8, 0);
    u64 bit = 0;
    for (u64 x : v)
        for (int b = 0; b < w; ++b, ++bit)
            if ((x >> b) & 1) data[bit >> 3] |= u8(1u << (bit & 7));
}

std::vector<u64> bitunpack(const Bytes& meta, const Bytes& data) {
    if (meta.size() != 5) throw std::runtime_error("Invalid meta size in bitpacked data");
    u32 n = meta[0] | (u32(meta[1]) << 8) | (u32(meta[2]) << 16) | (u32(meta[3]) << 24);
    int w = meta[4];
    std::vector<u64> v(n, 0);
    u64 bit = 0;
    for (u32 i = 0; i < n; ++i)
        for (int b = 0; b < w; ++b, ++bit)
            if (data.at(bit >> 3) & (1u << (bit & 7))) v[i] |= 1ull << b;
    return v;
}

// GolombRiceCoder<T>::pack (encoder/golomb_rice_encoder.hpp:92-148): one k per stream,
// k = floor(log2(mean)) (0 when all zero or mean < 1, capped at 62); q ones, a zero, then
// the k low bits, all LSB-first.  Empty input -> empty meta and data.
void gr_pack(const std::vector<u64>& v, Bytes& meta, Bytes& data) {
    meta.clear();
    data.clear();
    if (v.empty()) return;
    u64 sum = 0;
    bool zeros = true;
    for (u64 x : v) {
        if (x) zeros = false;
        sum += x;
    }
    u8 k = 0;
    if (!zeros) {
        double avg = static_cast<double>(sum) / v.size();
        k = avg < 1.0 ? 0 : static_cast<u8>(std::floor(std::log2(avg)));
    }
    if (k >= 63) k = 62;
    u32 n = static_cast<u32>(v.size());
    meta = {u8(n), u8(n >> 8), u8(n >> 16), u8(n >> 24), k};
    u64 bit = 0;
    auto put = [&](bool b) {
        if ((bit >> 3) >= data.size()) data.push_back(0);
        if (b) data[bit >> 3] |= u8(1u << (bit & 7));
        ++bit;
    };
    for (u64 x : v) {
        u64 q = x >> k;
        for (u64 i = 0; i < q; ++i) put(true);
        put(false);
        for (int b = 0; b < k; ++b) put((x >> b) & 1);
    }
}

std::vector<u64> gr_unpack(const Bytes& meta, const Bytes& data, u64 maxval) {
    if (meta.empty() && data.empty()) return {};
    if (meta.size() != 5) throw std::runtime_error("Invalid meta size in Golomb-Rice packed data");
    u32 n = meta[0] | (u32(meta[1]) << 8) | (u32(meta[2]) << 16) | (u32(meta[3]) << 24);
    if (n == 0) return {};
    u8 k = meta[4];
    if (k >= 63) throw std::runtime_error("Invalid k_param");
    std::vector<u64> v;
    v.reserve(n);
    u64 bit = 0, total = data.size() * 8ull;
    auto get = [&]() -> bool {
        if (bit >= total) throw std::out_of_range("Attempting to read beyond bitstream boundary");
        bool b = (data[bit >> 3] >> (bit & 7)) & 1;
        ++bit;
        return b;
    };
    for (u32 i = 0; i < n; ++i) {
        u64 q = 0;
        while (get()) ++q;
        u64 r = 0;
        for (int b = 0; b < k; ++b)
            if (get()) r |= 1ull << b;
        u64 val = q * (1ull << k) + r;
        if (val > maxval) throw std::runtime_error("Unpacked value exceeds capacity of target type T.");
        v.push_back(val);
    }
    return v;
}

// ---------------------------------------------------------------- Huffman -------------
// HuffmanEncoder<T> (encoder/huffman_encoder.hpp).  `Code` as in :251.
template <typename T>
struct Huff {
    struct Node {
        T sym{};
        u64 freq = 0;
        std::shared_ptr<Node> l, r;
    };
    struct Code {
        u32 bits;
        u8 len;
    };
    std::unordered_map<T, Code> table;
    bool eg = false;
    u8 egk = 0;

    static u64 to_u(T v) {
        if constexpr (std::is_signed<T>::value) {
            int64_t s = static_cast<int64_t>(v);
            return (static_cast<u64>(s) << 1) ^ static_cast<u64>(s >> 63);
        } else {
            return static_cast<u64>(v);
        }
    }
    static int blen(u64 v) {
        int l = v ? 64 - __builtin_clzll(v) : 0;
        return l ? l : 1;
    }
    // select_best_exp_golomb_k (:344-363)
    static u8 best_k(const std::vector<T>& d) {
        u64 best = std::numeric_limits<u64>::max();
        u8 bk = 0;
        for (u8 k = 0; k <= 16; ++k) {
            u64 cost = 0;
            for (T v : d) cost += static_cast<u64>(2 * blen((to_u(v) >> k) + 1) - 1 + k);
            if (cost < best) {
                best = cost;
                bk = k;
            }
        }
        return bk;
    }
    void walk(const std::shared_ptr<Node>& nd, u32 prefix, u8 len) {  // build_code (:269-281)
        if (!nd->l && !nd->r) {
            table[nd->sym] = len == 0 ? Code{0, 1} : Code{prefix, len};
            return;
        }
        walk(nd->l, prefix << 1, static_cast<u8>(len + 1));
        walk(nd->r, (prefix << 1) | 1u, static_cast<u8>(len + 1));
    }
    // build (:33-61) + build_from_freq (:91-123)
    void build(const std::vector<T>& d) {
        table.clear();
        if (d.empty()) return;
        std::unordered_map<T, u64> freq;
        for (T v : d) freq[v]++;
        double ent = 0.0;
        for (auto& kv : freq) {
            double p = double(kv.second) / d.size();
            ent -= p * std::log2(p);
        }
        if (ent > 10.0 || eg) {
            eg = true;
            egk = best_k(d);
            return;
        }
        from_freq(freq);
    }
    // build_from_freq (:91-123)
    void from_freq(const std::unordered_map<T, u64>& freq) {
        auto cmp = [](const std::shared_ptr<Node>& a, const std::shared_ptr<Node>& b) { return a->freq > b->freq; };
        std::priority_queue<std::shared_ptr<Node>, std::vector<std::shared_ptr<Node>>, decltype(cmp)> pq(cmp);
        for (auto& kv : freq) {
            auto n = std::make_shared<Node>();
            n->sym = kv.first;
            n->freq = kv.second;
            pq.push(n);
        }
        while (pq.size() > 1) {
            auto a = pq.top();
            pq.pop();
            auto b = pq.top();
            pq.pop();
            auto p = std::make_shared<Node>();
            p->freq = a->freq + b->freq;
            p->l = a;
            p->r = b;
            pq.push(p);
        }
        walk(pq.top(), 0u, 0);
    }
    // build_complete (:70-85): the data's frequencies, every missing value of [0, amax] with
    // frequency 1, built without the exp-Golomb switch.
    void build_complete(const std::vector<T>& d, T amax) {
        table.clear();
        eg = false;
        egk = 0;
        std::unordered_map<T, u64> freq;
        for (T v : d) freq[v]++;
        for (T s = 0; s <= amax; ++s) {
            if (freq.find(s) == freq.end()) freq[s] = 1;
            if (s == std::numeric_limits<T>::max()) break;
        }
        from_freq(freq);
    }
    // load_meta (:172-203): entries inserted in the meta's order.
    void load_meta(const Bytes& m) {
        table.clear();
        eg = false;
        egk = 0;
        size_t p = 0;
        if (m.size() >= 4 && m[0] == 0xE1 && m[1] == 0xC1 && m[2] == 0x01) {
            p = 4;
            if (m[3] == 0x01) {
                egk = m.size() > 4 ? m[4] : 0;
                eg = true;
                return;
            }
        }
        auto be32 = [&]() {
            if (p + 4 > m.size()) throw std::runtime_error("truncated Huffman meta");
            u32 v = (u32(m[p]) << 24) | (u32(m[p + 1]) << 16) | (u32(m[p + 2]) << 8) | u32(m[p + 3]);
            p += 4;
            return v;
        };
        const u32 count = be32();
        for (u32 i = 0; i < count; ++i) {
            if (p + sizeof(T) + 5 > m.size()) throw std::runtime_error("truncated Huffman meta");
            T sym;
            if constexpr (sizeof(T) == 8) {
                u64 v = 0;
                for (int k = 0; k < 8; ++k) v = (v << 8) | m[p++];
                sym = static_cast<T>(v);
            } else {
                std::memcpy(&sym, m.data() + p, sizeof(T));
                p += sizeof(T);
            }
            const u8 l = m[p++];
            const u32 b = be32();
            table[sym] = Code{b, l};
        }
    }
    // get_meta (:126-146): u32 BE count; per entry symbol (u64 BE, else native bytes),
    // u8 len, u32 BE bits.  exp-Golomb: E1 C1 01 01 k.
    Bytes meta() const {
        if (eg) return {0xE1, 0xC1, 0x01, 0x01, egk};
        Bytes o;
        auto be32 = [&](u32 v) {
            o.push_back(u8(v >> 24));
            o.push_back(u8(v >> 16));
            o.push_back(u8(v >> 8));
            o.push_back(u8(v));
        };
        be32(static_cast<u32>(table.size()));
        for (auto& kv : table) {
            if constexpr (sizeof(T) == 8) {
                for (int s = 56; s >= 0; s -= 8) o.push_back(u8(static_cast<u64>(kv.first) >> s));
            } else {
                T v = kv.first;
                const u8* b = reinterpret_cast<const u8*>(&v);
                o.insert(o.end(), b, b + sizeof(T));
            }
            o.push_back(kv.second.len);
            be32(kv.second.bits);
        }
        return o;
    }
    // encode (:150-170) and encode_exp_golomb (:365-396): MSB-first.
    Bytes encode(const std::vector<T>& d) const {
        Bytes o;
        if (eg) {
            u8 acc = 0, nb = 0;
            auto put = [&](unsigned b) {
                acc = u8((acc << 1) | (b & 1));
                if (++nb == 8) {
                    o.push_back(acc);
                    acc = 0;
                    nb = 0;
                }
            };
            for (T v : d) {
                u64 n = to_u(v), n1 = (n >> egk) + 1;
                int nb1 = blen(n1);
                for (int i = 0; i < nb1 - 1; ++i) put(0);
                for (int i = nb1 - 1; i >= 0; --i) put((n1 >> i) & 1);
                for (int i = 0; i < egk; ++i) put((n >> i) & 1);
            }
            if (nb) o.push_back(u8(acc << (8 - nb)));
            return o;
        }
        // Bit-serial form of the reference's 64-bit accumulator: the code is emitted as
        // `len` bits of `bits`, most significant first.
        u8 acc = 0, nb = 0;
        for (T v : d) {
            const Code& c = table.at(v);
            for (int i = c.len - 1; i >= 0; --i) {
                unsigned b = i < 32 ? (c.bits >> i) & 1 : 0;
                acc = u8((acc << 1) | b);
                if (++nb == 8) {
                    o.push_back(acc);
                    acc = 0;
                    nb = 0;
                }
            }
        }
        if (nb) o.push_back(u8(acc << (8 - nb)));
        return o;
    }
};

template <typename T>
T read_sym(const Bytes& m, size_t& p) {
    if constexpr (sizeof(T) == 8) {
        u64 v = 0;
        for (int k = 0; k < 8; ++k) v = (v << 8) | m.at(p++);
        return static_cast<T>(v);
    } else {
        T v;
        if (p + sizeof(T) > m.size()) throw std::runtime_error("truncated Huffman meta");
        std::memcpy(&v, m.data() + p, sizeof(T));
        p += sizeof(T);
        return v;
    }
}

// load_meta + decode (:172-243) and decode_exp_golomb (:398-442).
template <typename T>
std::vector<T> huff_decode(const Bytes& meta, const Bytes& data, u64 n) {
    std::vector<T> out;
    if (meta.size() >= 4 && meta[0] == 0xE1 && meta[1] == 0xC1 && meta[2] == 0x01 && meta[3] == 0x01) {
        u8 k = meta.size() > 4 ? meta[4] : 0;
        u64 bit = 0, total = data.size() * 8ull;
        auto get = [&](int& b) {
            if (bit >= total) return false;
            b = (data[bit >> 3] >> (7 - (bit & 7))) & 1;
            ++bit;
            return true;
        };
        while (out.size() < n) {
            int b = 0, z = 0;
            while (true) {
                if (!get(b)) return out;
                if (b == 0) ++z;
                else break;
            }
            u64 n1 = 1;
            for (int i = 0; i < z; ++i) {
                if (!get(b)) return out;
                n1 = (n1 << 1) | u64(b);
            }
            u64 hi = (n1 - 1) << k, lo = 0;
            for (int i = 0; i < k; ++i) {
                if (!get(b)) return out;
                lo |= u64(b) << i;
            }
            u64 v = hi | lo;
            if constexpr (std::is_signed<T>::value)
                out.push_back(static_cast<T>(static_cast<int64_t>((v >> 1) ^ (~(v & 1) + 1))));
            else
                out.push_back(static_cast<T>(v));
        }
        return out;
    }
    size_t p = 0;
    auto be32 = [&]() {
        if (p + 4 > meta.size()) throw std::runtime_error("truncated Huffman meta");
        u32 v = (u32(meta[p]) << 24) | (u32(meta[p + 1]) << 16) | (u32(meta[p + 2]) << 8) | u32(meta[p + 3]);
        p += 4;
        return v;
    };
    u32 cnt = be32();
    std::map<std::pair<u8, u32>, T> dec;
    std::vector<T> syms;
    for (u32 i = 0; i < cnt; ++i) {
        T s = read_sym<T>(meta, p);
        u8 len = meta.at(p++);
        u32 bits = be32();
        dec[{len, bits}] = s;
        syms.push_back(s);
    }
    std::set<T> distinct(syms.begin(), syms.end());
    if (distinct.size() == 1) {
        out.assign(n, *distinct.begin());
        return out;
    }
    u32 buf = 0;
    u8 blen = 0;
    for (u64 i = 0; i < data.size() * 8ull && out.size() < n; ++i) {
        buf = (buf << 1) | ((data[i >> 3] >> (7 - (i & 7))) & 1);
        ++blen;
        auto it = dec.find({blen, buf});
        if (it != dec.end()) {
            out.push_back(it->second);
            buf = 0;
            blen = 0;
        }
    }
    return out;
}

// ---------------------------------------------------------------- container -----------
struct Writer {
    Bytes b;
    template <typename V>
    void pod(V v) {
        const u8* p = reinterpret_cast<const u8*>(&v);
        b.insert(b.end(), p, p + sizeof(V));
    }
    // [u64 data_len][u64 meta_len][meta][data] (block_compressor.hpp:152-155)
    void stream(const Bytes& meta, const Bytes& data) {
        pod<u64>(data.size());
        pod<u64>(meta.size());
        b.insert(b.end(), meta.begin(), meta.end());
        b.insert(b.end(), data.begin(), data.end());
    }
};

struct Reader {
    const u8* p;
    const u8* end;
    template <typename V>
    V pod() {
        if (p + sizeof(V) > end) throw std::runtime_error("truncated container");
        V v;
        std::memcpy(&v, p, sizeof(V));
        p += sizeof(V);
        return v;
    }
    void stream(Bytes& meta, Bytes& data) {
        u64 dl = pod<u64>(), ml = pod<u64>();
        if (ml > u64(end - p) || dl > u64(end - p) - ml) throw std::runtime_error("truncated container");
        meta.assign(p, p + ml);
        p += ml;
        data.assign(p, p + dl);
        p += dl;
    }
};

// PForDeltaEncoder<T>::encode (encoder/p_for_delta_encoder.hpp:27-43), limit 254.
template <typename T>
void pfd(const std::vector<T>& v, std::vector<T>& sym, std::vector<u64>& patches) {
    sym.clear();
    patches.clear();
    sym.reserve(v.size());
    for (T x : v) {
        if (x > T(254)) {
            patches.push_back(x);
            sym.push_back(0);
        } else {
            sym.push_back(static_cast<T>(x + 1));
        }
    }
}

template <typename T>
void huff_stream(Writer& w, const std::vector<T>& sym) {
    Huff<T> h;
    h.build(sym);
    w.stream(h.meta(), h.encode(sym));
}

// Shared codebooks of compress_internal (composer/block_compressor.hpp:271-431): mode 1
// builds complete codebooks and records their metas, mode 2 loads the given metas.
struct Share {
    int mode = 0;
    Bytes rep_in, quad_in;    // mode 2
    Bytes rep_out, quad_out;  // mode 1
};

template <typename T>
void huff_stream_shared(Writer& w, const std::vector<T>& sym, Share& sh, bool repos) {
    Huff<T> h;
    if (sh.mode == 2) h.load_meta(repos ? sh.rep_in : sh.quad_in);
    else h.build_complete(sym, static_cast<T>(255));
    const Bytes m = h.meta();
    if (sh.mode == 1) (repos ? sh.rep_out : sh.quad_out) = m;
    w.stream(m, h.encode(sym));
}

struct Cell {
    i32 x, y, z;
};

// Sorted-record form of block_quantize (quantizer/block_quantizer.hpp:84-151).
struct Rec {
    u64 id, reid, ord;
};

void block_records(const std::vector<Cell>& cells, int rx, int ry, int rz, bool hil, std::vector<Rec>& rec) {
    const u64 B = 64;
    u64 nx = u64(rx) / (2 * B) + 1, ny = u64(ry) / (2 * B) + 1;
    (void)rz;
    rec.resize(cells.size());
    for (size_t i = 0; i < cells.size(); ++i) {
        u64 X = u64(int64_t(cells[i].x)), Y = u64(int64_t(cells[i].y)), Z = u64(int64_t(cells[i].z));
        u64 cx = X / B, dx = X % B, cy = Y / B, dy = Y % B, cz = Z / B, dz = Z % B;
        u64 id = (cx / 2) + (cy / 2) * nx + (cz / 2) * nx * ny;
        u64 m = morton(i32(dx), i32(dy), i32(dz));
        if (hil) m = m2h(m, 20);
        rec[i] = {id, m | ((cx & 1) << 60) | ((cy & 1) << 61) | ((cz & 1) << 62), i};
    }
    // Order: by id, then by reid (radix_sort + per-id std::sort, :33-76).  Records equal in
    // both keys are identical cells and the stream does not depend on their order.
    std::stable_sort(rec.begin(), rec.end(),
                     [](const Rec& a, const Rec& b) { return a.id != b.id ? a.id < b.id : a.reid < b.reid; });
}

struct Lcp {
    std::vector<u64> blkst, blkcnt, repos;
    std::vector<u8> quads;
};

// LCP stream construction (:117-149).
void lcp_streams(const std::vector<Rec>& rec, Lcp& m) {
    u64 prevId = ~0ull, prevQuad = 0, prevRe = 0;
    m.quads.resize(rec.size());
    m.repos.resize(rec.size());
    for (size_t j = 0; j < rec.size(); ++j) {
        u64 id = rec[j].id, quad = rec[j].reid >> 60, re = rec[j].reid & 0x0fffffffffffffffull;
        if (id != prevId) {
            m.blkst.push_back(id);
            m.blkcnt.push_back(0);
            prevId = id;
            prevQuad = 0;
            prevRe = 0;
        } else if (quad != prevQuad) {
            prevRe = 0;
        }
        m.blkcnt.back() += 1;
        m.quads[j] = u8(quad - prevQuad);
        m.repos[j] = re - prevRe;
        prevQuad = quad;
        prevRe = re;
    }
    if (m.blkst.empty()) {  // blknum starts at 1 (:117): one empty block for n == 0
        m.blkst.push_back(0);
        m.blkcnt.push_back(0);
    }
}

// Core compressor producing the pre-zstd container.
// BlockCompressor::compress (composer/block_compressor.hpp:39-222) and
// BlockCompressorRLE::compress (composer/block_compressor_rle.hpp:38-321).
Bytes compress_container(const float* xyz, u64 n, int quantizer, float l2, bool hil, bool rle, int thresh,
                         std::vector<u64>* order, Share* share = nullptr) {
    float off[3];
    std::vector<i32> q;
    std::vector<float> params;
    quantize_all(xyz, n, quantizer, l2, off, q, &params);
    std::vector<Cell> cells(n);
    for (u64 i = 0; i < n; ++i) cells[i] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};

    std::vector<int> cnts;
    if (rle) {
        // unordered_map dedup (:97-123): the stream only depends on the set of distinct
        // cells and their counts, so sort + unique stands in for the hash table.
        std::vector<u64> idx(n);
        for (u64 i = 0; i < n; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](u64 a, u64 b) {
            const Cell &A = cells[a], &B = cells[b];
            if (A.x != B.x) return A.x < B.x;
            if (A.y != B.y) return A.y < B.y;
            if (A.z != B.z) return A.z < B.z;
            return a < b;
        });
        std::vector<Cell> uc;
        for (u64 i = 0; i < n; ++i) {
            const Cell& c = cells[idx[i]];
            if (i == 0 || c.x != uc.back().x || c.y != uc.back().y || c.z != uc.back().z) {
                uc.push_back(c);
                cnts.push_back(1);
            } else {
                cnts.back()++;
            }
        }
        cells.swap(uc);
    }
    const u64 m = cells.size();

    Writer w;
    w.pod<u64>(m);
    w.pod<u64>(params.size());  // TO and cube have none, adaptive its three steps
    for (float v : params) w.pod<float>(v);
    int rx = 0, ry = 0, rz = 0;
    for (auto& c : cells) {
        rx = std::max(rx, c.x);
        ry = std::max(ry, c.y);
        rz = std::max(rz, c.z);
    }
    w.pod<i32>(rx);
    w.pod<i32>(ry);
    w.pod<i32>(rz);
    int mr = std::max({rx, ry, rz});
    bool direct = !share && mr < thresh;  // shared codebooks: always block mode
    w.pod<bool>(hil);
    w.pod<bool>(direct);
    std::vector<u64> perm(m);
    if (direct) {
        int bits = 0;
        for (int t = mr; t > 0; t >>= 1) ++bits;
        if (bits == 0) bits = 1;
        std::vector<std::pair<u64, u64>> e(m);
        for (u64 i = 0; i < m; ++i) {
            u64 mc = morton(cells[i].x, cells[i].y, cells[i].z);
            e[i] = {hil ? m2h(mc, bits) : mc, i};
        }
        std::sort(e.begin(), e.end());
        std::vector<u64> d(m);
        for (u64 i = 0; i < m; ++i) {
            d[i] = i == 0 ? e[0].first : e[i].first - e[i - 1].first;
            perm[i] = e[i].second;
        }
        std::vector<u64> sym, pat;
        pfd(d, sym, pat);
        Bytes gm, gd;
        gr_pack(pat, gm, gd);
        w.stream(gm, gd);
        huff_stream(w, sym);
    } else {
        std::vector<Rec> rec;
        block_records(cells, rx, ry, rz, hil, rec);
        for (u64 i = 0; i < m; ++i) perm[i] = rec[i].ord;
        Lcp L;
        lcp_streams(rec, L);
        for (size_t i = L.blkcnt.size() - 1; i > 0; --i) L.blkcnt[i] -= L.blkcnt[i - 1];
        for (size_t i = L.blkst.size() - 1; i > 0; --i) L.blkst[i] -= L.blkst[i - 1];
        Bytes bm, bd;
        bitpack(L.blkst, bm, bd);
        w.stream(bm, bd);
        bitpack(L.blkcnt, bm, bd);
        w.stream(bm, bd);
        std::vector<u64> sym, pat;
        pfd(L.repos, sym, pat);
        Bytes gm, gd;
        gr_pack(pat, gm, gd);
        w.stream(gm, gd);
        if (share) huff_stream_shared(w, sym, *share, true);
        else huff_stream(w, sym);
        std::vector<u8> qs;
        std::vector<u64> qp;
        pfd(L.quads, qs, qp);
        gr_pack(qp, gm, gd);  // GolombRiceCoder<uint8_t>: same bits for values < 256
        w.stream(gm, gd);
        if (share) huff_stream_shared(w, qs, *share, false);
        else huff_stream(w, qs);
    }
    if (rle) {
        std::vector<int> sc(m);
        for (u64 i = 0; i < m; ++i) sc[i] = cnts[perm[i]];
        // Counts stream (block_compressor_rle.hpp:290-308): build, measure, optionally
        // force exp-Golomb, then build again on the same encoder object.
        Huff<int> h;
        h.build(sc);
        Bytes m5 = h.meta(), c5 = h.encode(sc);
        if (static_cast<double>(m5.size()) > static_cast<double>(c5.size()) * 0.25) h.eg = true;
        h.build(sc);
        w.stream(h.meta(), h.encode(sc));
    }
    w.pod<float>(off[0]);
    w.pod<float>(off[1]);
    w.pod<float>(off[2]);
    if (order) *order = perm;
    return w.b;
}

// BlockDecompressor::decompress (composer/block_decompressor.hpp:31-192) and the RLE
// variant (composer/block_decompressor_rle.hpp:32-207), from the pre-zstd container.
std::vector<float> decompress_container(const Bytes& buf, int quantizer, float l2, bool rle) {
    Reader r{buf.data(), buf.data() + buf.size()};
    u64 n = r.pod<u64>();
    u64 np = r.pod<u64>();
    std::vector<float> params;
    for (u64 i = 0; i < np; ++i) params.push_back(r.pod<float>());
    if (quantizer == 2 && !rle && np < 3) throw std::runtime_error("adaptive container without its three steps");
    i32 rx = r.pod<i32>(), ry = r.pod<i32>(), rz = r.pod<i32>();
    bool hil = r.pod<bool>(), direct = r.pod<bool>();
    std::vector<Cell> cells(n);
    Bytes meta, data;
    if (direct) {
        r.stream(meta, data);
        auto pat = gr_unpack(meta, data, ~0ull);
        r.stream(meta, data);
        auto sym = huff_decode<u64>(meta, data, n);
        if (sym.size() < n) throw std::runtime_error("short Huffman stream");
        int mr = std::max({rx, ry, rz}), bits = 0;
        for (int t = mr; t > 0; t >>= 1) ++bits;
        if (bits == 0) bits = 1;
        u64 acc = 0, pi = 0;
        for (u64 i = 0; i < n; ++i) {
            u64 d = sym[i] == 0 ? pat.at(pi++) : sym[i] - 1;
            acc = i == 0 ? d : acc + d;
            u64 mc = hil ? h2m(acc, bits) : acc;
            cells[i] = {i32(gather3(mc)), i32(gather3(mc >> 1)), i32(gather3(mc >> 2))};
        }
    } else {
        r.stream(meta, data);
        auto blk = bitunpack(meta, data);
        r.stream(meta, data);
        auto cnt = bitunpack(meta, data);
        r.stream(meta, data);
        auto pat = gr_unpack(meta, data, ~0ull);
        r.stream(meta, data);
        auto sym = huff_decode<u64>(meta, data, n);
        r.stream(meta, data);
        auto qpat = gr_unpack(meta, data, 255);
        r.stream(meta, data);
        auto qsym = huff_decode<u8>(meta, data, n);
        if (sym.size() < n || qsym.size() < n) throw std::runtime_error("short Huffman stream");
        for (size_t i = 1; i < cnt.size(); ++i) cnt[i] += cnt[i - 1];
        for (size_t i = 1; i < blk.size(); ++i) blk[i] += blk[i - 1];
        const u64 B = 64;
        u64 nx = u64(rx) / (2 * B) + 1, ny = u64(ry) / (2 * B) + 1;
        u64 j = 0, pi = 0, qi = 0;
        for (size_t b = 0; b < blk.size(); ++b) {
            u64 pbx = (blk[b] % nx * 2) * B, pby = (blk[b] / nx % ny * 2) * B, pbz = (blk[b] / nx / ny * 2) * B;
            u64 pq = 0, pr = 0;
            for (u64 t = 0; t < cnt[b]; ++t, ++j) {
                if (j >= n) throw std::runtime_error("block counts exceed point count");
                u64 rep = sym[j] == 0 ? pat.at(pi++) : sym[j] - 1;
                u8 qd = qsym[j] == 0 ? u8(qpat.at(qi++)) : u8(qsym[j] - 1);
                if (qd != 0) pr = 0;
                u64 rj = rep + pr, qj = qd + pq;
                pr = rj;
                pq = qj;
                u64 mc = hil ? h2m(rj, 20) : rj;
                u64 ix = pbx + ((qj & 1) >> 0) * B + gather3(mc);
                u64 iy = pby + ((qj & 2) >> 1) * B + gather3(mc >> 1);
                u64 iz = pbz + ((qj & 4) >> 2) * B + gather3(mc >> 2);
                cells[j] = {i32(ix), i32(iy), i32(iz)};
            }
        }
        cells.resize(j);
    }
    std::vector<Cell> full;
    if (rle) {
        r.stream(meta, data);
        auto c = huff_decode<int>(meta, data, n);
        if (c.size() < cells.size()) throw std::runtime_error("short counts stream");
        for (size_t i = 0; i < cells.size(); ++i)
            for (int k = 0; k < c[i]; ++k) full.push_back(cells[i]);
    } else {
        full.swap(cells);
    }
    float off[3] = {r.pod<float>(), r.pod<float>(), r.pod<float>()};
    QConst k = make_const(quantizer, l2);
    std::vector<float> out(full.size() * 3);
    for (size_t i = 0; i < full.size(); ++i) {
        i32 c[3] = {full[i].x, full[i].y, full[i].z};
        float p[3];
        // BlockDecompressorRLE picks TO or else cube (block_decompressor_rle.hpp:189-196):
        // adaptive -rle containers are recovered with the cube quantizer there.
        if (quantizer == 1)
            recover_to(c, k, p);
        else if (quantizer == 2 && !rle)
            recover_adaptive(c, params.data(), p);
        else
            recover_cube(c, k, p);
        for (int d = 0; d < 3; ++d) out[3 * i + d] = p[d] + off[d];
    }
    return out;
}

template <typename V>
u8* dup(const V& v, u64* len) {
    *len = v.size() * sizeof(typename V::value_type);
    u8* p = static_cast<u8*>(std::malloc(*len ? *len : 1));
    if (*len) std::memcpy(p, v.data(), *len);
    return p;
}

}  // namespace

extern "C" {

void orc_free(void* p) { std::free(p); }

int orc_set_zstd_library(const char* path) {
    std::snprintf(g_zstd_path, sizeof(g_zstd_path), "%s", path);
    return zstd_load() ? 0 : 1;
}

// Pre-zstd container (zstd_level < 0) or the zstd level-3 frame (zstd_level = 3).
int orc_compress(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, int rle, int direct_threshold,
                 int zstd_level, uint8_t** out, uint64_t* out_len, uint64_t* order_out) {
    try {
        std::vector<u64> order;
        Bytes c = compress_container(xyz, n, quantizer, l2, hilbert != 0, rle != 0, direct_threshold,
                                     order_out ? &order : nullptr);
        if (order_out)
            for (size_t i = 0; i < order.size(); ++i) order_out[i] = order[i];
        if (zstd_level >= 0) {
            if (!zstd_load()) return 3;
            Bytes z(g_zstd.compressBound(c.size()));
            size_t zs = g_zstd.compress(z.data(), z.size(), c.data(), c.size(), zstd_level);
            if (g_zstd.isError(zs)) return 4;
            z.resize(zs);
            c.swap(z);
        }
        *out = dup(c, out_len);
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_compress: %s\n", e.what());
        return 1;
    }
}

// fit_profile / compress_with_profile (composer/block_compressor.hpp:241-256), -normal; the
// profile in serialize_profile's layout (composer/block_encoding_profile.hpp:34-48).
static int finish_frame(Bytes& c, int zstd_level, uint8_t** out, uint64_t* out_len) {
    if (zstd_level >= 0) {
        if (!zstd_load()) return 3;
        Bytes z(g_zstd.compressBound(c.size()));
        size_t zs = g_zstd.compress(z.data(), z.size(), c.data(), c.size(), zstd_level);
        if (g_zstd.isError(zs)) return 4;
        z.resize(zs);
        c.swap(z);
    }
    *out = dup(c, out_len);
    return 0;
}

int orc_fit_profile(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, int zstd_level, uint8_t** out,
                    uint64_t* out_len, uint8_t** prof, uint64_t* prof_len) {
    try {
        Share sh;
        sh.mode = 1;
        Bytes c = compress_container(xyz, n, quantizer, l2, hilbert != 0, false, 1024, nullptr, &sh);
        Bytes blob;
        for (const Bytes* m : {&sh.rep_out, &sh.quad_out}) {
            const u32 len = static_cast<u32>(m->size());
            for (int b = 0; b < 4; ++b) blob.push_back(u8(len >> (8 * b)));
            blob.insert(blob.end(), m->begin(), m->end());
        }
        *prof = dup(blob, prof_len);
        return finish_frame(c, zstd_level, out, out_len);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_fit_profile: %s\n", e.what());
        return 1;
    }
}

int orc_compress_with_profile(const float* xyz, uint64_t n, int quantizer, float l2, int hilbert, const uint8_t* prof,
                              uint64_t prof_len, int zstd_level, uint8_t** out, uint64_t* out_len) {
    try {
        Share sh;
        sh.mode = 2;
        uint64_t p = 0;
        for (Bytes* m : {&sh.rep_in, &sh.quad_in}) {
            if (p + 4 > prof_len) throw std::runtime_error("malformed profile");
            const u32 len = u32(prof[p]) | (u32(prof[p + 1]) << 8) | (u32(prof[p + 2]) << 16) | (u32(prof[p + 3]) << 24);
            p += 4;
            if (len > prof_len - p) throw std::runtime_error("malformed profile");
            m->assign(prof + p, prof + p + len);
            p += len;
        }
        if (sh.rep_in.empty() || sh.quad_in.empty()) throw std::runtime_error("empty profile");
        Bytes c = compress_container(xyz, n, quantizer, l2, hilbert != 0, false, 1024, nullptr, &sh);
        return finish_frame(c, zstd_level, out, out_len);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_compress_with_profile: %s\n", e.what());
        return 1;
    }
}

int orc_decompress(const uint8_t* buf, uint64_t len, int is_zstd, int quantizer, float l2, int rle, float** xyz,
                   uint64_t* n_out) {
    try {
        Bytes c(buf, buf + len);
        if (is_zstd) {
            if (!zstd_load()) return 3;
            unsigned long long fs = g_zstd.frameContentSize(buf, len);
            if (fs >= (0ULL - 2)) return 4;
            Bytes raw(fs);
            size_t ds = g_zstd.decompress(raw.data(), fs, buf, len);
            if (g_zstd.isError(ds) || ds != fs) return 4;
            c.swap(raw);
        }
        auto v = decompress_container(c, quantizer, l2, rle != 0);
        *n_out = v.size() / 3;
        *xyz = reinterpret_cast<float*>(dup(v, &len));
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "orc_decompress: %s\n", e.what());
        return 1;
    }
}

// Stage entry points used by the parity tests.
int orc_quantize(const float* xyz, uint64_t n, int quantizer, float l2, float* offset3, int32_t* q_out) {
    std::vector<i32> q;
    quantize_all(xyz, n, quantizer, l2, offset3, q);
    std::memcpy(q_out, q.data(), q.size() * 4);
    return 0;
}

int orc_recover(const int32_t* q, uint64_t n, int quantizer, float l2, const float* off, float* out) {
    QConst k = make_const(quantizer, l2);
    for (uint64_t i = 0; i < n; ++i) {
        float p[3];
        if (quantizer == 1)
            recover_to(q + 3 * i, k, p);
        else
            recover_cube(q + 3 * i, k, p);
        for (int d = 0; d < 3; ++d) out[3 * i + d] = p[d] + off[d];
    }
    return 0;
}

uint64_t orc_morton(int x, int y, int z) { return morton(x, y, z); }
void orc_m2h(const uint64_t* in, uint64_t n, unsigned iter, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = m2h(in[i], iter);
}
void orc_h2m(const uint64_t* in, uint64_t n, unsigned iter, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = h2m(in[i], iter);
}
void orc_hilbert_tables(uint8_t* child_h2m64) {
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) child_h2m64[8 * i + j] = tables().childH2M[i][j];
}

// Sorted (id, reid) records of block_quantize for lattice cells.
int orc_block_records(const int32_t* q, uint64_t n, int rx, int ry, int rz, int hilbert, uint64_t* id_out,
                      uint64_t* reid_out) {
    std::vector<Cell> cells(n);
    for (uint64_t i = 0; i < n; ++i) cells[i] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
    std::vector<Rec> rec;
    block_records(cells, rx, ry, rz, hilbert != 0, rec);
    for (uint64_t i = 0; i < n; ++i) {
        id_out[i] = rec[i].id;
        reid_out[i] = rec[i].reid;
    }
    return 0;
}

int orc_huffman(int kind, const void* data, uint64_t n, int force_eg, uint8_t** meta, uint64_t* ml, uint8_t** enc,
                uint64_t* el) {
    auto run = [&](auto tag) {
        using T = decltype(tag);
        const T* d = static_cast<const T*>(data);
        std::vector<T> v(d, d + n);
        Huff<T> h;
        h.eg = force_eg != 0;
        h.build(v);
        *meta = dup(h.meta(), ml);
        *enc = dup(h.encode(v), el);
    };
    if (kind == 0) run(u64{});
    else if (kind == 1) run(u8{});
    else run(int{});
    return 0;
}

int orc_gr_pack(const uint64_t* data, uint64_t n, uint8_t** meta, uint64_t* ml, uint8_t** enc, uint64_t* el) {
    Bytes m, d;
    gr_pack(std::vector<u64>(data, data + n), m, d);
    *meta = dup(m, ml);
    *enc = dup(d, el);
    return 0;
}

int orc_bitpack(const uint64_t* data, uint64_t n, uint8_t** meta, uint64_t* ml, uint8_t** enc, uint64_t* el) {
    try {
        Bytes m, d;
        bitpack(std::vector<u64>(data, data + n), m, d);
        *meta = dup(m, ml);
        *enc = dup(d, el);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

}  // extern "C"
