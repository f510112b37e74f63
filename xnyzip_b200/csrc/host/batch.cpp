// Batches of independent clouds (xnyz_batch_*): a pool of host threads, each driving its own
// context and CUDA stream, so that the host-side libzstd frames (single-threaded per frame,
// as in composer/utils.hpp:35-53) of different clouds run in parallel and overlap the GPU
// stages of the others.  Each cloud goes through exactly the per-cloud entry points, so
// every frame is byte-identical to a lone xnyz_compress call.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/xnyz.h"

namespace xnyz {
xnyz_status set_last_error(xnyz_status s, const std::string& msg);
}

struct xnyz_batch {
    int device = 0;
    std::vector<xnyz_ctx*> ctx;
};

namespace {

// Runs f(ctx, i) for every i in `order` on the pool; returns the first failure by index.
template <class F>
xnyz_status run_pool(xnyz_batch* b, const std::vector<uint64_t>& order, F&& f, xnyz_status* item_status) {
    const uint64_t count = order.size();
    std::vector<xnyz_status> st(count, XNYZ_OK);
    std::vector<std::string> msg(count);
    std::atomic<uint64_t> next{0};
    auto work = [&](size_t w) {
        for (;;) {
            const uint64_t k = next.fetch_add(1);
            if (k >= count) break;
            const uint64_t i = order[k];
            st[i] = f(b->ctx[w], i);
            if (st[i] != XNYZ_OK) msg[i] = xnyz_last_error();
        }
    };
    const size_t nt = static_cast<size_t>(std::min<uint64_t>(b->ctx.size(), count));
    std::vector<std::thread> th;
    th.reserve(nt);
    for (size_t w = 1; w < nt; ++w) th.emplace_back(work, w);
    if (nt) work(0);
    for (auto& t : th) t.join();
    xnyz_status ret = XNYZ_OK;
    for (uint64_t i = 0; i < count; ++i) {
        if (item_status) item_status[i] = st[i];
        if (ret == XNYZ_OK && st[i] != XNYZ_OK) {
            ret = st[i];
            xnyz::set_last_error(st[i], "cloud " + std::to_string(i) + ": " + msg[i]);
        }
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

}  // extern "C"
