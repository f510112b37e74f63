// Batches of independent clouds (xnyz_batch_*): a pool of host threads, each driving its own
// context and CUDA stream, so that the host-side libzstd frames (single-threaded per frame,
// as in composer/utils.hpp:35-53) of different clouds run in parallel and overlap the GPU
// stages of the others.  Each cloud goes through exactly the per-cloud entry points, so
// every frame is byte-identical to a lone xnyz_compress call.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/xnyz.h"

namespace xnyz {
xnyz_status set_last_error(xnyz_status s, const std::string& msg);
}

// Size classes of the device round trip: by point count, powers of four from 16K.
constexpr int kClasses = 6;
inline int size_class(uint64_t n) {
    int b = 0;
    for (uint64_t v = n; v; v >>= 1) ++b;
    const int c = (b - 14) / 2;
    return c < 0 ? 0 : (c >= kClasses ? kClasses - 1 : c);
}

struct xnyz_batch {
    int device = 0;
    std::vector<xnyz_ctx*> ctx;
    int class_workers[kClasses] = {0, 0, 0, 0, 0, 0};  // 0: all workers
};

namespace {

// Runs f(ctx, i) for every i in `order` on the pool; returns the first failure by index.
template <class F>
xnyz_status run_pool(xnyz_batch* b, const std::vector<uint64_t>& order, F&& f, xnyz_status* item_status,
                     size_t max_workers = 0) {
    const uint64_t count = order.size();
    std::vector<xnyz_status> st(count, XNYZ_OK);
    std::vector<std::string> msg(count);
    std::atomic<uint64_t> next{0};
    auto work = [&](size_t w) {
        for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= count) break;
            const uint64_t i = order[k];
            st[k] = f(b->ctx[w], i);
            if (st[k] != XNYZ_OK) msg[k] = xnyz_last_error();
        }
    };
    size_t nt = static_cast<size_t>(std::min<uint64_t>(b->ctx.size(), count));
    if (max_workers && max_workers < nt) nt = max_workers;
    std::vector<std::thread> th;
    th.reserve(nt);
    for (size_t w = 1; w < nt; ++w) th.emplace_back(work, w);
    if (nt) work(0);
    for (auto& t : th) t.join();
    // statuses are kept per position in `order` (which may be a subset of the clouds)
    xnyz_status ret = XNYZ_OK;
    uint64_t first_bad = 0;
    for (uint64_t k = 0; k < count; ++k) {
        if (item_status) item_status[order[k]] = st[k];
        if (st[k] != XNYZ_OK && (ret == XNYZ_OK || order[k] < order[first_bad])) {
            ret = st[k];
            first_bad = k;
        }
    }
    if (ret != XNYZ_OK)
        xnyz::set_last_error(ret, "cloud " + std::to_string(order[first_bad]) + ": " + msg[first_bad]);
    return ret;
}

// Device round trip of clouds `idx` (compress into the worker's context, then decompress
// the device container), one size class at a time, largest class first, each class with its
// tuned number of concurrent workers.
xnyz_status roundtrip(xnyz_batch* b, const std::vector<uint64_t>& idx, const float* const* xyz, const uint64_t* n,
                      const xnyz_params* params, uint64_t* out_len, uint64_t* out_n, xnyz_status* item_status,
                      const int* workers_per_class) {
    std::vector<uint64_t> cls[kClasses];
    for (uint64_t i : idx) cls[size_class(n[i])].push_back(i);
    xnyz_status ret = XNYZ_OK;
    for (int c = kClasses - 1; c >= 0; --c) {
        if (cls[c].empty()) continue;
        std::stable_sort(cls[c].begin(), cls[c].end(), [&](uint64_t a, uint64_t bb) { return n[a] > n[bb]; });
        const xnyz_status s = run_pool(
            b, cls[c],
            [&](xnyz_ctx* cx, uint64_t i) {
                const uint8_t* dc = nullptr;
                uint64_t dl = 0;
                xnyz_status r = xnyz_compress_device(cx, xyz[i], n[i], &params[i], &dc, &dl, nullptr);
                if (r != XNYZ_OK) return r;
                out_len[i] = dl;
                const float* dp = nullptr;
                r = xnyz_decompress_device(cx, dc, dl, params[i].quantizer, params[i].l2_bound, params[i].rle, &dp,
                                           &out_n[i]);
                return r;
            },
            item_status, static_cast<size_t>(workers_per_class[c]));
        if (ret == XNYZ_OK) ret = s;
    }
    return ret;
}

// Largest first (longest-processing-time order), ties by index.
template <class Size>
std::vector<uint64_t> largest_first(uint64_t count, Size&& size) {
    std::vector<uint64_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return size(a) > size(b); });
    return order;
}

}  // namespace

extern "C" {

xnyz_status xnyz_batch_set_block_mode(xnyz_batch* b, int mode) {
    if (!b) return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null batch");
    for (xnyz_ctx* c : b->ctx) {
        const xnyz_status s = xnyz_set_block_mode(c, mode);
        if (s != XNYZ_OK) return s;
    }
    return XNYZ_OK;
}

xnyz_status xnyz_batch_create(xnyz_batch** out, int device, int workers) {
    if (!out) return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null batch pointer");
    *out = nullptr;
    if (workers <= 0) workers = static_cast<int>(std::min(32u, std::max(1u, std::thread::hardware_concurrency())));
    auto* b = new xnyz_batch();
    b->device = device;
    for (int w = 0; w < workers; ++w) {
        xnyz_ctx* c = nullptr;
        const xnyz_status s = xnyz_create(&c, device, nullptr);
        if (s != XNYZ_OK) {
            const std::string m = xnyz_last_error();
            xnyz_batch_destroy(b);
            return xnyz::set_last_error(s, m);
        }
        b->ctx.push_back(c);
    }
    *out = b;
    return XNYZ_OK;
}

xnyz_status xnyz_batch_destroy(xnyz_batch* b) {
    if (!b) return XNYZ_OK;
    for (xnyz_ctx* c : b->ctx) xnyz_destroy(c);
    delete b;
    return XNYZ_OK;
}

int xnyz_batch_workers(const xnyz_batch* b) { return b ? static_cast<int>(b->ctx.size()) : 0; }

xnyz_status xnyz_batch_roundtrip_device(xnyz_batch* b, uint64_t count, const float* const* xyz, const uint64_t* n,
                                        const xnyz_params* params, uint64_t* out_len, uint64_t* out_n,
                                        xnyz_status* item_status) {
    if (!b || (count && (!xyz || !n || !params || !out_len || !out_n)))
        return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null argument");
    std::vector<uint64_t> idx(count);
    for (uint64_t i = 0; i < count; ++i) {
        idx[i] = i;
        out_len[i] = out_n[i] = 0;
    }
    return roundtrip(b, idx, xyz, n, params, out_len, out_n, item_status, b->class_workers);
}

xnyz_status xnyz_batch_autotune(xnyz_batch* b, uint64_t count, const float* const* xyz, const uint64_t* n,
                                const xnyz_params* params, int* class_workers) {
    if (!b || (count && (!xyz || !n || !params))) return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null argument");
    std::vector<uint64_t> cls[kClasses];
    for (uint64_t i = 0; i < count; ++i) cls[size_class(n[i])].push_back(i);
    std::vector<uint64_t> len(count), nout(count);
    const int wmax = static_cast<int>(b->ctx.size());
    for (int c = 0; c < kClasses; ++c) {
        b->class_workers[c] = 0;
        if (cls[c].empty()) continue;
        // a sample of the class: up to 4 x the workers, at most 64M points
        std::vector<uint64_t> sample;
        uint64_t pts = 0;
        for (uint64_t i : cls[c]) {
            if (sample.size() >= static_cast<size_t>(4 * wmax) || pts + n[i] > (64ull << 20)) break;
            sample.push_back(i);
            pts += n[i];
        }
        if (sample.empty()) sample.push_back(cls[c][0]);
        double best = -1.0;
        int best_w = wmax;
        for (int w = 1; w <= wmax; w *= 2) {
            int wc[kClasses];
            for (int k = 0; k < kClasses; ++k) wc[k] = w;
            xnyz_status s = roundtrip(b, sample, xyz, n, params, len.data(), nout.data(), nullptr, wc);  // warm-up
            if (s != XNYZ_OK) return s;
            const auto t0 = std::chrono::steady_clock::now();
            s = roundtrip(b, sample, xyz, n, params, len.data(), nout.data(), nullptr, wc);
            if (s != XNYZ_OK) return s;
            const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            const double rate = static_cast<double>(pts) / std::max(dt, 1e-9);
            if (rate > best * 1.02) {  // more workers only for a clear gain
                best = rate;
                best_w = w;
            }
        }
        b->class_workers[c] = best_w;
    }
    if (class_workers)
        for (int c = 0; c < kClasses; ++c) class_workers[c] = b->class_workers[c];
    return XNYZ_OK;
}

xnyz_status xnyz_batch_compress(xnyz_batch* b, uint64_t count, const float* const* xyz, const uint64_t* n,
                                int xyz_is_device, const xnyz_params* params, int use_zstd, uint8_t** out,
                                uint64_t* out_len, xnyz_status* item_status) {
    if (!b || (count && (!xyz || !n || !params || !out || !out_len)))
        return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null argument");
    for (uint64_t i = 0; i < count; ++i) {
        out[i] = nullptr;
        out_len[i] = 0;
    }
    const auto order = largest_first(count, [&](uint64_t i) { return n[i]; });
    return run_pool(
        b, order,
        [&](xnyz_ctx* c, uint64_t i) {
            return xnyz_compress(c, xyz[i], n[i], xyz_is_device, &params[i], use_zstd, &out[i], &out_len[i], nullptr,
                                 nullptr);
        },
        item_status);
}

xnyz_status xnyz_batch_decompress(xnyz_batch* b, uint64_t count, const uint8_t* const* in, const uint64_t* in_len,
                                  int is_zstd, const int* quantizer, const float* l2_bound, const int* rle,
                                  float* const* xyz, const uint64_t* capacity, uint64_t* n, xnyz_status* item_status) {
    if (!b || (count && (!in || !in_len || !quantizer || !l2_bound || !rle || !xyz || !capacity || !n)))
        return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null argument");
    for (uint64_t i = 0; i < count; ++i) n[i] = 0;
    const auto order = largest_first(count, [&](uint64_t i) { return in_len[i]; });
    return run_pool(
        b, order,
        [&](xnyz_ctx* c, uint64_t i) {
            return xnyz_decompress_into(c, in[i], in_len[i], is_zstd, quantizer[i], l2_bound[i], rle[i], xyz[i],
                                        capacity[i], &n[i]);
        },
        item_status);
}

xnyz_status xnyz_batch_roundtrip(xnyz_batch* b, uint64_t count, const float* const* xyz, const uint64_t* n,
                                 const xnyz_params* params, uint8_t** frame, uint64_t* frame_len, float* const* out,
                                 xnyz_status* item_status) {
    if (!b || (count && (!xyz || !n || !params || !frame || !frame_len || !out)))
        return xnyz::set_last_error(XNYZ_ERR_INVALID_ARG, "null argument");
    for (uint64_t i = 0; i < count; ++i) {
        frame[i] = nullptr;
        frame_len[i] = 0;
    }
    const auto order = largest_first(count, [&](uint64_t i) { return n[i]; });
    return run_pool(
        b, order,
        [&](xnyz_ctx* c, uint64_t i) {
            xnyz_status s = xnyz_compress(c, xyz[i], n[i], 0, &params[i], 1, &frame[i], &frame_len[i], nullptr,
                                          nullptr);
            if (s != XNYZ_OK) return s;
            uint64_t got = 0;
            s = xnyz_decompress_into(c, frame[i], frame_len[i], 1, params[i].quantizer, params[i].l2_bound,
                                     params[i].rle, out[i], n[i], &got);
            if (s == XNYZ_OK && got != n[i])
                return xnyz::set_last_error(XNYZ_ERR_BAD_STREAM, "round trip changed the point count");
            return s;
        },
        item_status);
}

}  // extern "C"
