/* C++ drop-in for the reference's composer classes, over the C ABI of libxnyz.so.
 *
 * A caller of the reference library keeps its code: the class names, constructors, method
 * signatures and exception types below are those of the XnYZip composer headers
 *   BlockCompressor<T>        composer/block_compressor.hpp:31-39, 241-256
 *   BlockCompressorRLE<T>     composer/block_compressor_rle.hpp:30-38, 341-348
 *   BlockDecompressor<T>      composer/block_decompressor.hpp:25-31
 *   BlockDecompressorRLE<T>   composer/block_decompressor_rle.hpp:26-32, 221-230, 339-341
 *   QUANTIZER_TYPE            composer/utils.hpp:55-59
 *   BlockEncodingProfile, serialize_profile, deserialize_profile
 *                             composer/block_encoding_profile.hpp:17-72
 * and every compute stage runs on the GPU.  Outputs are byte-identical to the reference's
 * (the zstd frame of compress(), the points of decompress()).
 *
 * Points are Eigen::RowVector<T, 3> as in the reference; define XNYZ_COMPAT_NO_EIGEN before
 * including this header to use the plain 12-byte Vec3 below instead.  Only T = float is
 * supported (the reference instantiates nothing else).  Each object owns one xnyz context
 * (device 0, default stream) and is movable, not copyable.
 *
 * Exceptions, as the reference throws them: std::runtime_error for zstd failures, damaged or
 * truncated containers and an empty profile; std::invalid_argument for bad arguments (the
 * reference's BitPacker on empty input); std::runtime_error for every other failure (the
 * message is xnyz_last_error()).
 *
 * Link: -L<dir of libxnyz.so> -lxnyz -Wl,-rpath,<dir>. */
#ifndef XNYZ_COMPAT_HPP
#define XNYZ_COMPAT_HPP

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "xnyz.h"

#ifndef XNYZ_COMPAT_NO_EIGEN
#include <Eigen/Dense>
#endif

namespace XnYZip {

#ifndef XNYZ_COMPAT_NO_EIGEN
template <typename T>
using Vec3 = Eigen::RowVector<T, 3>;
using Cell3 = Eigen::RowVector3i;
#else
template <typename T>
struct Vec3 {
    T v[3];
    Vec3() : v{T(0), T(0), T(0)} {}
    Vec3(T x, T y, T z) : v{x, y, z} {}
    T& operator[](int i) { return v[i]; }
    const T& operator[](int i) const { return v[i]; }
    T x() const { return v[0]; }
    T y() const { return v[1]; }
    T z() const { return v[2]; }
    T* data() { return v; }
    const T* data() const { return v; }
};
using Cell3 = Vec3<int>;
#endif

enum class QUANTIZER_TYPE { CUBE, TRUNCATED_OCTAHEDRON, ADAPTIVE };

struct BlockEncodingProfile {
    std::vector<uint8_t> repos_huff_meta;
    std::vector<uint8_t> quads_huff_meta;
    bool valid() const { return !repos_huff_meta.empty() && !quads_huff_meta.empty(); }
};

/* [u32 LE length][repos meta][u32 LE length][quads meta], the reference's flat layout. */
inline std::vector<uint8_t> serialize_profile(const BlockEncodingProfile& p) {
    std::vector<uint8_t> out;
    auto put = [&](const std::vector<uint8_t>& m) {
        const uint32_t n = static_cast<uint32_t>(m.size());
        for (int k = 0; k < 4; ++k) out.push_back(static_cast<uint8_t>(n >> (8 * k)));
        out.insert(out.end(), m.begin(), m.end());
    };
    put(p.repos_huff_meta);
    put(p.quads_huff_meta);
    return out;
}

inline BlockEncodingProfile deserialize_profile(const std::vector<uint8_t>& in) {
    BlockEncodingProfile p;
    size_t pos = 0;
    auto get = [&](std::vector<uint8_t>& m) {
        if (pos + 4 > in.size()) throw std::runtime_error("deserialize_profile: truncated length");
        uint32_t n = 0;
        for (int k = 0; k < 4; ++k) n |= static_cast<uint32_t>(in[pos + k]) << (8 * k);
        pos += 4;
        if (n > in.size() - pos) throw std::runtime_error("deserialize_profile: truncated meta");
        m.assign(in.begin() + static_cast<std::ptrdiff_t>(pos), in.begin() + static_cast<std::ptrdiff_t>(pos + n));
        pos += n;
    };
    get(p.repos_huff_meta);
    get(p.quads_huff_meta);
    return p;
}

namespace compat_detail {

inline void check(xnyz_status s) {
    if (s == XNYZ_OK) return;
    const char* msg = xnyz_last_error();
    const std::string m = msg ? msg : "xnyz error";
    if (s == XNYZ_ERR_INVALID_ARG) throw std::invalid_argument(m);
    throw std::runtime_error(m);
}

/* malloc'd library buffer -> vector, released either way */
template <typename V, typename P>
V take(P* p, uint64_t count) {
    V v;
    if (count) v.assign(p, p + count);
    xnyz_free(p);
    return v;
}

class Ctx {
   public:
    Ctx() { check(xnyz_create(&c_, 0, nullptr)); }
    ~Ctx() {
        if (c_) xnyz_destroy(c_);
    }
    Ctx(const Ctx&) = delete;
    Ctx& operator=(const Ctx&) = delete;
    Ctx(Ctx&& o) noexcept : c_(o.c_) { o.c_ = nullptr; }
    Ctx& operator=(Ctx&& o) noexcept {
        std::swap(c_, o.c_);
        return *this;
    }
    xnyz_ctx* get() const { return c_; }

   private:
    xnyz_ctx* c_ = nullptr;
};

template <typename T>
const float* xyz_of(const std::vector<Vec3<T>>& pts) {
    static_assert(std::is_same<T, float>::value, "only float points are supported");
    static_assert(sizeof(Vec3<T>) == 3 * sizeof(float), "points must be 12 contiguous bytes");
    return pts.empty() ? nullptr : pts.data()->data();
}

/* compress() reorders its argument into the container's point order (block_compressor.hpp:141-144) */
template <typename T>
void apply_order(std::vector<Vec3<T>>& pts, const std::vector<uint64_t>& order) {
    std::vector<Vec3<T>> out(pts.size());
    for (size_t i = 0; i < pts.size(); ++i) out[i] = pts[order[i]];
    pts.swap(out);
}

template <typename T>
std::vector<Vec3<T>> to_points(float* xyz, uint64_t n) {
    std::vector<Vec3<T>> out(n);
    if (n) std::memcpy(static_cast<void*>(out.data()), xyz, 12 * n);
    xnyz_free(xyz);
    return out;
}

}  // namespace compat_detail

template <typename T>
class BlockCompressor {
   public:
    BlockCompressor(QUANTIZER_TYPE quantizer_type, float l2_bound, bool is_debugging = false, int direct_threshold = 1024)
        : p_{static_cast<int>(quantizer_type), l2_bound, 0, 0, direct_threshold} {
        (void)is_debugging;
    }

    auto compress(std::vector<Vec3<T>>& points, bool curve_type) -> std::vector<uint8_t> {
        p_.hilbert = curve_type ? 1 : 0;
        std::vector<uint64_t> order(points.size());
        uint8_t* out = nullptr;
        uint64_t len = 0;
        compat_detail::check(xnyz_compress(ctx_.get(), compat_detail::xyz_of(points), points.size(), 0, &p_, 1, &out,
                                           &len, order.data(), nullptr));
        compat_detail::apply_order(points, order);
        return compat_detail::take<std::vector<uint8_t>>(out, len);
    }

    auto fit_profile(std::vector<Vec3<T>>& points, bool curve_type)
        -> std::pair<std::vector<uint8_t>, BlockEncodingProfile> {
        p_.hilbert = curve_type ? 1 : 0;
        std::vector<uint64_t> order(points.size());
        uint8_t *out = nullptr, *prof = nullptr;
        uint64_t len = 0, plen = 0;
        compat_detail::check(xnyz_fit_profile(ctx_.get(), compat_detail::xyz_of(points), points.size(), 0, &p_, 1, &out,
                                              &len, order.data(), &prof, &plen));
        compat_detail::apply_order(points, order);
        auto bytes = compat_detail::take<std::vector<uint8_t>>(out, len);
        return {std::move(bytes), deserialize_profile(compat_detail::take<std::vector<uint8_t>>(prof, plen))};
    }

    auto compress_with_profile(std::vector<Vec3<T>>& points, bool curve_type, const BlockEncodingProfile& profile)
        -> std::vector<uint8_t> {
        if (!profile.valid()) throw std::runtime_error("compress_with_profile: empty profile");
        p_.hilbert = curve_type ? 1 : 0;
        const std::vector<uint8_t> blob = serialize_profile(profile);
        std::vector<uint64_t> order(points.size());
        uint8_t* out = nullptr;
        uint64_t len = 0;
        compat_detail::check(xnyz_compress_with_profile(ctx_.get(), compat_detail::xyz_of(points), points.size(), 0,
                                                        &p_, blob.data(), blob.size(), 1, &out, &len, order.data()));
        compat_detail::apply_order(points, order);
        return compat_detail::take<std::vector<uint8_t>>(out, len);
    }

   private:
    compat_detail::Ctx ctx_;
    xnyz_params p_;
};

template <typename T>
class BlockCompressorRLE {
   public:
    BlockCompressorRLE(QUANTIZER_TYPE quantizer_type, float l2_bound, bool is_debugging = false,
                       int direct_threshold = 1024)
        : p_{static_cast<int>(quantizer_type), l2_bound, 0, 1, direct_threshold} {
        (void)is_debugging;
    }

    auto compress(std::vector<Vec3<T>>& points, bool curve_type) -> std::vector<uint8_t> {
        p_.hilbert = curve_type ? 1 : 0;
        uint8_t* out = nullptr;
        uint64_t len = 0;
        compat_detail::check(xnyz_compress(ctx_.get(), compat_detail::xyz_of(points), points.size(), 0, &p_, 1, &out,
                                           &len, nullptr, nullptr));
        return compat_detail::take<std::vector<uint8_t>>(out, len);
    }

    auto encode_cells_with_counts(std::vector<Cell3>& cells, std::vector<int>& counts, int range_x, int range_y,
                                  int range_z, Vec3<T> offset, bool curve_type) -> std::vector<uint8_t> {
        if (cells.size() != counts.size())
            throw std::runtime_error("encode_cells_with_counts: cells and counts size mismatch");
        static_assert(sizeof(Cell3) == 12, "cells must be 12 contiguous bytes");
        const int32_t ranges[3] = {range_x, range_y, range_z};
        const float off[3] = {offset[0], offset[1], offset[2]};
        uint8_t* out = nullptr;
        uint64_t len = 0;
        compat_detail::check(xnyz_encode_cells(ctx_.get(), cells.empty() ? nullptr : cells.data()->data(),
                                               counts.data(), cells.size(), 0, ranges, off, curve_type ? 1 : 0, 1,
                                               &out, &len));
        return compat_detail::take<std::vector<uint8_t>>(out, len);
    }

   private:
    compat_detail::Ctx ctx_;
    xnyz_params p_;
};

template <typename T>
class BlockDecompressor {
   public:
    BlockDecompressor(QUANTIZER_TYPE quantizer_type, float l2_bound, bool is_debugging = false)
        : q_(static_cast<int>(quantizer_type)), l2_(l2_bound) {
        (void)is_debugging;
    }

    auto decompress(const std::vector<uint8_t>& compressed_data) -> std::vector<Vec3<T>> {
        float* xyz = nullptr;
        uint64_t n = 0;
        compat_detail::check(
            xnyz_decompress(ctx_.get(), compressed_data.data(), compressed_data.size(), 1, q_, l2_, 0, &xyz, &n));
        return compat_detail::to_points<T>(xyz, n);
    }

   private:
    compat_detail::Ctx ctx_;
    int q_;
    float l2_;
};

template <typename T>
class BlockDecompressorRLE {
   public:
    struct DecodedCellTable {
        std::vector<Cell3> cells;
        std::vector<int> counts;
        std::vector<T> params;
        Vec3<T> offset;
        int range_x = 0, range_y = 0, range_z = 0;
        bool is_hilbert = false;
    };

    BlockDecompressorRLE(QUANTIZER_TYPE quantizer_type, float l2_bound, bool is_debugging = false)
        : q_(static_cast<int>(quantizer_type)), l2_(l2_bound) {
        (void)is_debugging;
    }

    auto decompress(const std::vector<uint8_t>& compressed_data) -> std::vector<Vec3<T>> {
        float* xyz = nullptr;
        uint64_t n = 0;
        compat_detail::check(
            xnyz_decompress(ctx_.get(), compressed_data.data(), compressed_data.size(), 1, q_, l2_, 1, &xyz, &n));
        return compat_detail::to_points<T>(xyz, n);
    }

    auto decompress_to_cells(const std::vector<uint8_t>& compressed_data) -> DecodedCellTable {
        int32_t *cells = nullptr, *counts = nullptr;
        uint64_t n = 0;
        float off[3];
        int32_t ranges[3];
        int hil = 0;
        compat_detail::check(xnyz_decompress_to_cells(ctx_.get(), compressed_data.data(), compressed_data.size(), 1,
                                                      &cells, &counts, &n, off, ranges, &hil));
        DecodedCellTable t;
        t.cells.resize(n);
        if (n) std::memcpy(static_cast<void*>(t.cells.data()), cells, 12 * n);
        xnyz_free(cells);
        t.counts = compat_detail::take<std::vector<int>>(counts, n);
        t.offset = Vec3<T>(off[0], off[1], off[2]);
        t.range_x = ranges[0];
        t.range_y = ranges[1];
        t.range_z = ranges[2];
        t.is_hilbert = hil != 0;
        return t;
    }

    auto expand_cells_to_points(const DecodedCellTable& table) -> std::vector<Vec3<T>> {
        const float off[3] = {table.offset[0], table.offset[1], table.offset[2]};
        float* xyz = nullptr;
        uint64_t n = 0;
        compat_detail::check(xnyz_expand_cells(ctx_.get(), table.cells.empty() ? nullptr : table.cells.data()->data(),
                                               table.counts.data(), table.cells.size(), q_, l2_, off, &xyz, &n));
        return compat_detail::to_points<T>(xyz, n);
    }

   private:
    compat_detail::Ctx ctx_;
    int q_;
    float l2_;
};

}  // namespace XnYZip

#endif  // XNYZ_COMPAT_HPP
