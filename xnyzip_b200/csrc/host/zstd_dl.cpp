#include "zstd_dl.h"

#include <dlfcn.h>

#include <atomic>
#include <cstdlib>
#include <mutex>

#ifndef XNYZ_DEFAULT_ZSTD
#define XNYZ_DEFAULT_ZSTD ""
#endif

namespace xnyz {
namespace {

struct Api {
    unsigned (*version)(void) = nullptr;
    size_t (*bound)(size_t) = nullptr;
    size_t (*compress)(void*, size_t, const void*, size_t, int) = nullptr;
    size_t (*decompress)(void*, size_t, const void*, size_t) = nullptr;
    unsigned long long (*content_size)(const void*, size_t) = nullptr;
    unsigned (*is_error)(size_t) = nullptr;
    const char* (*error_name)(size_t) = nullptr;
    // explicit contexts: ZSTD_compressCCtx / ZSTD_decompressDCtx give the same bytes as
    // ZSTD_compress / ZSTD_decompress (which build and free a context per call)
    void* (*create_cctx)(void) = nullptr;
    size_t (*free_cctx)(void*) = nullptr;
    size_t (*compress_cctx)(void*, void*, size_t, const void*, size_t, int) = nullptr;
    void* (*create_dctx)(void) = nullptr;
    size_t (*free_dctx)(void*) = nullptr;
    size_t (*decompress_dctx)(void*, void*, size_t, const void*, size_t) = nullptr;
    void* handle = nullptr;
};

Api g_api;
std::mutex g_mu;
std::atomic<bool> g_loaded{false};

// One compression and one decompression context per host thread, kept for the thread's
// lifetime (the batch workers compress thousands of frames each).
struct ThreadContexts {
    void* c = nullptr;
    void* d = nullptr;
    ~ThreadContexts() {
        if (c && g_api.free_cctx) g_api.free_cctx(c);
        if (d && g_api.free_dctx) g_api.free_dctx(d);
    }
};
thread_local ThreadContexts t_ctx;
constexpr unsigned kWantVersion = 10507;  // 1.5.7

bool load_locked(const char* path, std::string& err) {
    if (g_api.handle) return true;
    std::string p;
    if (path && *path) p = path;
    else if (const char* e = std::getenv("XNYZ_ZSTD_LIBRARY")) p = e;
    else p = XNYZ_DEFAULT_ZSTD;
    if (p.empty()) {
        err = "libzstd 1.5.7 location unknown (set XNYZ_ZSTD_LIBRARY)";
        return false;
    }
    void* h = dlopen(p.c_str(), RTLD_NOW | RTLD_LOCAL);
    if (!h) {
        err = std::string("cannot load ") + p + ": " + dlerror();
        return false;
    }
    Api a;
    a.version = reinterpret_cast<unsigned (*)(void)>(dlsym(h, "ZSTD_versionNumber"));
    a.bound = reinterpret_cast<size_t (*)(size_t)>(dlsym(h, "ZSTD_compressBound"));
    a.compress = reinterpret_cast<size_t (*)(void*, size_t, const void*, size_t, int)>(dlsym(h, "ZSTD_compress"));
    a.decompress = reinterpret_cast<size_t (*)(void*, size_t, const void*, size_t)>(dlsym(h, "ZSTD_decompress"));
    a.content_size = reinterpret_cast<unsigned long long (*)(const void*, size_t)>(dlsym(h, "ZSTD_getFrameContentSize"));
    a.is_error = reinterpret_cast<unsigned (*)(size_t)>(dlsym(h, "ZSTD_isError"));
    a.error_name = reinterpret_cast<const char* (*)(size_t)>(dlsym(h, "ZSTD_getErrorName"));
    a.create_cctx = reinterpret_cast<void* (*)(void)>(dlsym(h, "ZSTD_createCCtx"));
    a.free_cctx = reinterpret_cast<size_t (*)(void*)>(dlsym(h, "ZSTD_freeCCtx"));
    a.compress_cctx =
        reinterpret_cast<size_t (*)(void*, void*, size_t, const void*, size_t, int)>(dlsym(h, "ZSTD_compressCCtx"));
    a.create_dctx = reinterpret_cast<void* (*)(void)>(dlsym(h, "ZSTD_createDCtx"));
    a.free_dctx = reinterpret_cast<size_t (*)(void*)>(dlsym(h, "ZSTD_freeDCtx"));
    a.decompress_dctx =
        reinterpret_cast<size_t (*)(void*, void*, size_t, const void*, size_t)>(dlsym(h, "ZSTD_decompressDCtx"));
    if (!a.version || !a.bound || !a.compress || !a.decompress || !a.content_size || !a.is_error || !a.error_name) {
        err = p + " lacks the zstd entry points";
        dlclose(h);
        return false;
    }
    if (a.version() != kWantVersion) {
        err = p + " is libzstd " + std::to_string(a.version()) + ", the container format needs 1.5.7 (10507)";
        dlclose(h);
        return false;
    }
    a.handle = h;
    g_api = a;
    g_loaded.store(true, std::memory_order_release);
    return true;
}

}  // namespace

bool zstd_load(const char* path, std::string& err) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_api.handle && path && *path) {
        // already loaded: keep the first library (functions are process-wide)
        return true;
    }
    return load_locked(path, err);
}

bool zstd_available(std::string& err) {
    if (g_loaded.load(std::memory_order_acquire)) return true;
    std::lock_guard<std::mutex> lk(g_mu);
    return load_locked(nullptr, err);
}

size_t zstd_bound(size_t n) { return g_api.bound ? g_api.bound(n) : 0; }

bool zstd_compress_into(const uint8_t* src, size_t n, int level, uint8_t* dst, size_t cap, size_t& written,
                        std::string& err) {
    if (!zstd_available(err)) return false;
    if (!t_ctx.c && g_api.create_cctx && g_api.compress_cctx) t_ctx.c = g_api.create_cctx();
    const size_t r = t_ctx.c ? g_api.compress_cctx(t_ctx.c, dst, cap, src, n, level)
                             : g_api.compress(dst, cap, src, n, level);
    if (g_api.is_error(r)) {
        err = g_api.error_name(r);
        return false;
    }
    written = r;
    return true;
}

bool zstd_compress(const uint8_t* src, size_t n, int level, std::vector<uint8_t>& out, std::string& err) {
    if (!zstd_available(err)) return false;
    out.resize(g_api.bound(n));
    size_t w = 0;
    if (!zstd_compress_into(src, n, level, out.data(), out.size(), w, err)) return false;
    out.resize(w);
    return true;
}

bool zstd_content_size(const uint8_t* src, size_t n, uint64_t& size, std::string& err) {
    if (!zstd_available(err)) return false;
    const unsigned long long s = g_api.content_size(src, n);
    if (s == (0ULL - 2)) {
        err = "Not a zstd frame";
        return false;
    }
    if (s == (0ULL - 1)) {
        err = "Original size unknown";
        return false;
    }
    size = s;
    return true;
}

bool zstd_decompress(const uint8_t* src, size_t n, uint8_t* dst, uint64_t dst_size, std::string& err) {
    if (!zstd_available(err)) return false;
    if (!t_ctx.d && g_api.create_dctx && g_api.decompress_dctx) t_ctx.d = g_api.create_dctx();
    const size_t r = t_ctx.d ? g_api.decompress_dctx(t_ctx.d, dst, dst_size, src, n)
                             : g_api.decompress(dst, dst_size, src, n);
    if (g_api.is_error(r)) {
        err = g_api.error_name(r);
        return false;
    }
    if (r != dst_size) {
        err = "Decompressed size mismatch";
        return false;
    }
    return true;
}

}  // namespace xnyz
