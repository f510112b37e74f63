// C ABI and host orchestration of the B200 XnYZip path (declared in include/xnyz.h).
//
// Compress (BlockCompressor{,RLE}<float>::compress, composer/block_compressor.hpp:39-222,
// composer/block_compressor_rle.hpp:38-321), every stage on the GPU:
//   bbox -> quantize + ranges -> [host: mode, key layout] -> keys (+ digit histograms)
//   -> LSD radix sort -> units (dedup, LCP deltas, PFor, histograms) -> count / block stats
//   -> [host: Huffman codebooks from histograms, Golomb-Rice k, bit widths]
//   -> bit-pack / Golomb-Rice / Huffman / exp-Golomb encoders -> container -> zstd (host).
// Decompress (BlockDecompressor{,RLE}<float>::decompress): zstd (host) -> header (host)
//   -> bit-unpack + prefix sums -> parallel Golomb-Rice / Huffman / exp-Golomb decoding
//   -> fused LCP recovery, PFor decode, expansion, recover and unshift.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/xnyz.h"
#include "host/codebook.h"
#include "host/hilbert_tables.h"
#include "host/zstd_dl.h"
#include "kernels.h"

using namespace xnyz;
using namespace xnyz::dev;

namespace {

thread_local std::string g_last_error;

xnyz_status fail(xnyz_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

#define CUDA_TRY(expr)                                                                               \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? XNYZ_ERR_OOM : XNYZ_ERR_CUDA,              \
                        std::string(#expr) + ": " + cudaGetErrorString(e_));                         \
    } while (0)

#define TRY(expr)                          \
    do {                                   \
        xnyz_status s_ = (expr);           \
        if (s_ != XNYZ_OK) return s_;      \
    } while (0)

constexpr size_t kAlign = 256;
// First 8 bytes of an extended container ("XNYZBX01"): the reference container follows,
// except that the repos / SFC-delta stream is block-coded (k_blocks.cu).
constexpr uint64_t kExtMagic = 0x313058425a594e58ull;
inline size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }
inline uint64_t cdiv(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
inline int bitlen(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

// Fixed-size device state of a context (counters, histograms, code tables, tables).
struct Small {
    PointStats stats;
    unsigned long long counters[8];
    unsigned long long hist_rep[256];
    uint32_t first_rep[256];
    unsigned long long hist_quad[256];
    uint32_t first_quad[256];
    unsigned long long cnt_hist[kCountDense];
    uint32_t cnt_first[kCountDense];
    uint32_t over_n;
    uint32_t err;
    uint32_t fallback[8];
    uint32_t maxrun[8];
    unsigned long long max2[2];
    unsigned long long totals[8];
    unsigned long long codewords[8];
    unsigned long long count_total;
    unsigned long long ext_bits;      // extended container: block payload bits
    unsigned long long ext_fallback;  // extended container: blocks searched exhaustively
    double ext_sum;                   // extended container: sum of the stream (global mode)
    uint32_t tile_counters[64];
    uint32_t sort_hist[8 * 256];
    ByteCodes codes[2];
    uint8_t hil_fwd[256];
    uint8_t hil_inv[256];
    float offset_in[4];
};

// A growable device arena, carved per call.
struct Arena {
    char* base = nullptr;
    size_t cap = 0;
};

struct Plan {
    size_t total = 0;
    size_t add(size_t bytes) {
        const size_t o = align_up(total);
        total = o + align_up(bytes ? bytes : 1);
        return o;
    }
};

}  // namespace

struct xnyz_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    Small* d_small = nullptr;
    Small* h_small = nullptr;  // pinned mirror
    Arena arena;
    unsigned long long* sort_status = nullptr;
    size_t sort_status_cap = 0;  // entries
    uint32_t sort_epoch = 0;
    uint8_t* h_stage = nullptr;  // pinned staging for containers
    size_t h_stage_cap = 0;
    uint8_t* d_container = nullptr;  // device container returned by xnyz_compress_device
    size_t d_container_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Side streams for independent streams of one container (the entropy coders and
    // decoders run concurrently); forked from and joined back into `stream` by events.
    static constexpr int kSide = 4;
    cudaStream_t side[kSide] = {};
    cudaEvent_t fork_ev = nullptr;
    cudaEvent_t join_ev[kSide] = {};
    // stage profiling (xnyz_profile / xnyz_profile_read); serial: side-stream work is issued
    // on the context's stream so that every stage's events time that stage alone
    bool prof = false;
    bool serial = false;
    struct ProfRec {
        const char* name;
        cudaEvent_t a, b;
        uint64_t launches;
        double bytes;
    };
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::map<std::string, std::pair<double, uint64_t>> host_ms;  // host phase wall time, calls
    // extended container (block parameters of the repos / SFC-delta stream)
    int block_mode = XNYZ_BLOCKS_OFF;
    // shared codebooks (fit_profile / compress_with_profile): 0 off, 1 fit (complete
    // codebooks, the profile of the call in share_out), 2 use share_rep / share_quad
    int share_mode = 0;
    std::vector<uint8_t> share_rep, share_quad, share_out;
    float* d_model = nullptr;      // predictor parameters (kParamCount FP32)
    float fallback_conf = 0.5f;    // learned mode: blocks below this confidence are searched
    xnyz_block_info last_blocks{};
    const unsigned long long* last_repval = nullptr;  // rep values of the last extended compress
    uint64_t last_repval_n = 0;
};

namespace {

xnyz_status ensure_arena(xnyz_ctx* c, size_t bytes) {
    if (c->arena.cap >= bytes) return XNYZ_OK;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->arena.base) cudaFree(c->arena.base);
    c->arena.base = nullptr;
    c->arena.cap = 0;
    const size_t want = align_up(bytes + bytes / 8, 1 << 20);
    CUDA_TRY(cudaMalloc(&c->arena.base, want));
    c->arena.cap = want;
    return XNYZ_OK;
}

xnyz_status ensure_host_stage(xnyz_ctx* c, size_t bytes) {
    if (c->h_stage_cap >= bytes) return XNYZ_OK;
    if (c->h_stage) cudaFreeHost(c->h_stage);
    c->h_stage = nullptr;
    c->h_stage_cap = 0;
    const size_t want = align_up(bytes + bytes / 8, 1 << 20);
    CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&c->h_stage), want, cudaHostAllocDefault));
    c->h_stage_cap = want;
    return XNYZ_OK;
}

cudaEvent_t pool_event(xnyz_ctx* c) {
    if (c->ev_used == c->ev_pool.size()) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// Brackets one stage's kernel launches with CUDA events on the context's stream when
// profiling is on.  `launches` counts the kernels, `bytes` their algorithmic traffic.
struct Prof {
    xnyz_ctx* c;
    const char* name;
    uint64_t launches;
    double bytes;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    Prof(xnyz_ctx* cc, const char* nm, uint64_t l, double b) : Prof(cc, nm, l, b, cc->stream) {}
    Prof(xnyz_ctx* cc, const char* nm, uint64_t l, double b, cudaStream_t on)
        : c(cc), name(nm), launches(l), bytes(b), s(on) {
        if (c->prof && (a = pool_event(c))) cudaEventRecord(a, s);
    }
    void end() {
        if (!c->prof || !a) return;
        cudaEvent_t e = pool_event(c);
        if (e) {
            cudaEventRecord(e, s);
            c->prof_recs.push_back(xnyz_ctx::ProfRec{name, a, e, launches, bytes});
        }
        a = nullptr;
    }
    ~Prof() { end(); }
};

// Wall time of a host phase (including the device work it waits for) when profiling.
struct HostPhase {
    xnyz_ctx* c;
    const char* name;
    std::chrono::steady_clock::time_point t0;
    bool open = true;
    HostPhase(xnyz_ctx* cc, const char* nm) : c(cc), name(nm), t0(std::chrono::steady_clock::now()) {}
    void end() {
        if (!open) return;
        open = false;
        if (!c->prof) return;
        auto& e = c->host_ms[name];
        e.first += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        e.second += 1;
    }
    ~HostPhase() { end(); }
};

template <typename T>
T* at(xnyz_ctx* c, size_t off) {
    return reinterpret_cast<T*>(c->arena.base + off);
}

#define SMALL_FIELD(c, f) (&(c)->d_small->f)

xnyz_status memset_small(xnyz_ctx* c, size_t off, size_t bytes, int v) {
    CUDA_TRY(cudaMemsetAsync(reinterpret_cast<char*>(c->d_small) + off, v, bytes, c->stream));
    return XNYZ_OK;
}

xnyz_status fetch_small(xnyz_ctx* c, size_t off, size_t bytes) {
    CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(c->h_small) + off, reinterpret_cast<char*>(c->d_small) + off,
                             bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return XNYZ_OK;
}

// Side stream k (the context's own stream when profiling serially).
inline cudaStream_t side(xnyz_ctx* c, int k) { return c->serial ? c->stream : c->side[k]; }

// Side stream k starts after the work queued so far on the context's stream.
xnyz_status fork_sides(xnyz_ctx* c) {
    CUDA_TRY(cudaEventRecord(c->fork_ev, c->stream));
    for (int k = 0; k < xnyz_ctx::kSide; ++k) CUDA_TRY(cudaStreamWaitEvent(c->side[k], c->fork_ev, 0));
    return XNYZ_OK;
}

// The context's stream continues after all work queued on the side streams.
xnyz_status join_sides(xnyz_ctx* c) {
    for (int k = 0; k < xnyz_ctx::kSide; ++k) {
        CUDA_TRY(cudaEventRecord(c->join_ev[k], c->side[k]));
        CUDA_TRY(cudaStreamWaitEvent(c->stream, c->join_ev[k], 0));
    }
    return XNYZ_OK;
}

// The device error word as last copied to the host.
xnyz_status device_errors(xnyz_ctx* c) {
    const uint32_t e = c->h_small->err;
    if (e & 1u) return fail(XNYZ_ERR_TIMEOUT, "a bounded device wait expired");
    if (e & 2u) return fail(XNYZ_ERR_BAD_STREAM, "malformed bit stream");
    if (e & 4u) return fail(XNYZ_ERR_BAD_STREAM, "stream content exceeds its declared sizes");
    if (e & 8u) return fail(XNYZ_ERR_TIMEOUT, "a scatter position fell outside its array after a wait expired");
    return XNYZ_OK;
}

xnyz_status check_device_errors(xnyz_ctx* c) {
    TRY(fetch_small(c, offsetof(Small, err), sizeof(uint32_t)));
    return device_errors(c);
}

QuantParams make_quant(int quantizer, float l2) {
    QuantParams q{};
    q.quantizer = quantizer;
    const double k = quantizer == 1 ? 5.0 : 3.0;
    // 2 * l2 in float, divided by sqrt(k) in double, stored as float (the reference's
    // `pt / (2 * TRUNC_OCT_SCALE_ / sqrt(k))` with Eigen's scalar conversion).
    q.div = static_cast<float>(static_cast<double>(2.0f * l2) / std::sqrt(k));
    q.s = l2;
    q.rdiv = static_cast<float>(std::sqrt(k));
    return q;
}

uint64_t spread3_host(uint32_t v) {
    uint64_t r = 0;
    for (int b = 0; b < 21; ++b) r |= static_cast<uint64_t>((v >> b) & 1u) << (3 * b);
    return r;
}

// The length shared by every codeword of a code table (len[s] = 0: symbol absent) when it is
// 1..24 bits, else 0.
int fixed_code_len(const uint8_t* len, size_t count) {
    int l = 0;
    for (size_t s = 0; s < count; ++s) {
        if (!len[s]) continue;
        if (!l) l = len[s];
        else if (len[s] != l) return 0;
    }
    return l >= 1 && l <= 24 ? l : 0;
}

// ---------------------------------------------------------------- sort ------------------
struct SortBufs {
    unsigned long long* keys[2];
    uint32_t* vals[2];
};

// Sorts keys (and payload) over `passes` 8-bit digits whose histograms are in hist (already
// filled).  Returns the index of the buffer holding the result.
xnyz_status radix_sort(xnyz_ctx* c, SortBufs& b, uint64_t n, int passes, uint32_t* d_hist, int& result) {
    result = 0;
    if (passes == 0 || n <= 1) return XNYZ_OK;
    const uint64_t tiles = cdiv(n, kSortTile);
    const size_t need = tiles * 256;
    if (c->sort_status_cap < need) {
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        if (c->sort_status) cudaFree(c->sort_status);
        c->sort_status = nullptr;
        const size_t want = need + need / 4 + 4096;
        CUDA_TRY(cudaMalloc(&c->sort_status, want * sizeof(unsigned long long)));
        CUDA_TRY(cudaMemsetAsync(c->sort_status, 0, want * sizeof(unsigned long long), c->stream));
        c->sort_status_cap = want;
        c->sort_epoch = 0;
    }
    if (c->sort_epoch + passes >= 16383) {
        CUDA_TRY(cudaMemsetAsync(c->sort_status, 0, c->sort_status_cap * sizeof(unsigned long long), c->stream));
        c->sort_epoch = 0;
    }
    launch_sort_offsets(d_hist, passes, c->stream);
    TRY(memset_small(c, offsetof(Small, tile_counters), sizeof(uint32_t) * 8, 0));
    int cur = 0;
    for (int p = 0; p < passes; ++p) {
        const uint32_t epoch = ++c->sort_epoch;
        Prof pr(c, "sort_pass", 1, (b.vals[0] ? 24.0 : 16.0) * n);
        launch_sort_pass(b.keys[cur], b.keys[cur ^ 1], b.vals[cur], b.vals[cur ^ 1], n, 8 * p, d_hist + 256 * p,
                         c->sort_status, epoch, SMALL_FIELD(c, tile_counters[p]), SMALL_FIELD(c, err), c->stream);
        cur ^= 1;
    }
    CUDA_TRY(cudaGetLastError());
    result = cur;
    return XNYZ_OK;
}

// ---------------------------------------------------------------- container --------------

// The container as an ordered list of pieces: header bytes kept on the host (a few KB) and
// stream payloads left in device memory until the container is assembled where it is needed.
struct Container {
    struct Piece {
        size_t off;        // offset in the container
        size_t len;
        size_t blob_off;   // host piece: offset in `blob`
        const void* dsrc;  // device piece: source (nullptr for host pieces)
    };
    std::vector<uint8_t> blob;  // all host bytes, in container order
    std::vector<Piece> pieces;
    size_t size = 0;
    void host_bytes(const void* p, size_t n) {
        if (!n) return;
        if (!pieces.empty() && !pieces.back().dsrc) {
            pieces.back().len += n;
        } else {
            pieces.push_back(Piece{size, n, blob.size(), nullptr});
        }
        const uint8_t* b = static_cast<const uint8_t*>(p);
        blob.insert(blob.end(), b, b + n);
        size += n;
    }
    template <typename V>
    void pod(V v) {
        host_bytes(&v, sizeof(V));
    }
    // [u64 data_len][u64 meta_len][meta][data]  (block_compressor.hpp:152-155)
    void stream(const std::vector<uint8_t>& meta, const void* ddata, size_t data_bytes) {
        pod<uint64_t>(data_bytes);
        pod<uint64_t>(meta.size());
        host_bytes(meta.data(), meta.size());
        if (data_bytes) {
            pieces.push_back(Piece{size, data_bytes, 0, ddata});
            size += data_bytes;
        }
    }
    // A stream whose data is several parts: device memory, or zero bytes where ptr is null.
    void stream_parts(const std::vector<uint8_t>& meta, std::initializer_list<std::pair<const void*, size_t>> parts) {
        size_t total = 0;
        for (const auto& pr : parts) total += pr.second;
        pod<uint64_t>(total);
        pod<uint64_t>(meta.size());
        host_bytes(meta.data(), meta.size());
        for (const auto& pr : parts) {
            if (!pr.second) continue;
            if (pr.first) {
                pieces.push_back(Piece{size, pr.second, 0, pr.first});
                size += pr.second;
            } else {
                const std::vector<uint8_t> z(pr.second, 0);
                host_bytes(z.data(), z.size());
            }
        }
    }
    // Assemble into host memory (device pieces copied asynchronously on `st`).
    cudaError_t to_host(uint8_t* dst, cudaStream_t st) const {
        for (const Piece& pc : pieces) {
            if (pc.dsrc) {
                const cudaError_t e = cudaMemcpyAsync(dst + pc.off, pc.dsrc, pc.len, cudaMemcpyDeviceToHost, st);
                if (e != cudaSuccess) return e;
            } else {
                std::memcpy(dst + pc.off, blob.data() + pc.blob_off, pc.len);
            }
        }
        return cudaSuccess;
    }
    // Assemble into device memory; host pieces are staged through `stage` (pinned, >= blob).
    cudaError_t to_device(uint8_t* dst, uint8_t* stage, cudaStream_t st) const {
        std::memcpy(stage, blob.data(), blob.size());
        for (const Piece& pc : pieces) {
            const cudaError_t e =
                pc.dsrc ? cudaMemcpyAsync(dst + pc.off, pc.dsrc, pc.len, cudaMemcpyDeviceToDevice, st)
                        : cudaMemcpyAsync(dst + pc.off, stage + pc.blob_off, pc.len, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
};

std::vector<uint8_t> le5(uint32_t n, uint8_t b) {
    return {static_cast<uint8_t>(n), static_cast<uint8_t>(n >> 8), static_cast<uint8_t>(n >> 16),
            static_cast<uint8_t>(n >> 24), b};
}

struct CompressOut {
    Container cont;
    xnyz_compress_info info{};
    uint32_t* d_order = nullptr;  // -normal: input index per container position
};

// One chained-scan channel set in the arena.
struct LB {
    size_t flag, agg, inc;
    uint64_t tiles;
};
LB plan_lb(Plan& pl, uint64_t tiles, int channels, int agg_words_per_tile = 1, int inc_words_per_tile = 1) {
    LB l;
    l.tiles = tiles;
    l.flag = pl.add(sizeof(uint32_t) * tiles * channels);
    l.agg = pl.add(sizeof(unsigned long long) * tiles * channels * agg_words_per_tile);
    l.inc = pl.add(sizeof(unsigned long long) * tiles * channels * inc_words_per_tile);
    return l;
}
LookBackState lb_state(xnyz_ctx* c, const LB& l) {
    return LookBackState{at<uint32_t>(c, l.flag), at<unsigned long long>(c, l.agg), at<unsigned long long>(c, l.inc)};
}
xnyz_status lb_clear(xnyz_ctx* c, const LB& l, int channels) {
    CUDA_TRY(cudaMemsetAsync(at<uint32_t>(c, l.flag), 0, sizeof(uint32_t) * l.tiles * channels, c->stream));
    return XNYZ_OK;
}

// Arena layout of the compress path up to the encoder outputs (depends on n only).
struct CPlan {
    uint64_t tiles;
    size_t o_k0, o_k1, o_v0, o_v1, o_rep, o_quad, o_patch, o_blkid, o_blkunit, o_unitpos, o_counts, o_over_v,
        o_over_u, o_dblk, o_dcnt;
    LB lb_units, lb_enc;
    size_t o_repval = 0, o_xw = 0, o_xk = 0, o_xoff = 0, o_xcost = 0, o_xfeat = 0, o_xconf = 0, o_xflag = 0;
    size_t total;
};
CPlan make_cplan(uint64_t n, bool want_order, size_t reserved, bool ext) {
    CPlan c{};
    c.tiles = cdiv(n, kSortTile);
    Plan pl;
    pl.total = reserved;
    c.o_k0 = pl.add(8 * n);
    c.o_k1 = pl.add(8 * n);
    c.o_v0 = want_order ? pl.add(4 * n) : 0;
    c.o_v1 = want_order ? pl.add(4 * n) : 0;
    c.o_rep = pl.add(n);
    c.o_quad = pl.add(n);
    c.o_patch = pl.add(8 * n);
    c.o_blkid = pl.add(8 * n);
    c.o_blkunit = pl.add(4 * n);
    c.o_unitpos = pl.add(4 * n + 4);
    c.o_counts = pl.add(4 * n);
    c.o_over_v = pl.add(4 * n);
    c.o_over_u = pl.add(4 * n);
    c.o_dblk = pl.add(8 * n);
    c.o_dcnt = pl.add(8 * n);
    c.lb_units = plan_lb(pl, c.tiles, 3);
    c.lb_enc = plan_lb(pl, c.tiles, 4);
    if (ext) {
        const uint64_t nb = cdiv(n, kParamBlock);
        c.o_repval = pl.add(8 * n);
        c.o_xw = pl.add(nb);
        c.o_xk = pl.add(nb);
        c.o_xoff = pl.add(8 * nb);
        c.o_xcost = pl.add(4 * nb);
        c.o_xfeat = pl.add(4ull * kParamFeatures * nb);
        c.o_xconf = pl.add(8 * nb);
        c.o_xflag = pl.add(nb);
    }
    c.total = pl.total;
    return c;
}
// Typical encoder output space (grown on demand when a stream is larger).
size_t encoder_reserve(uint64_t n) { return 4 * n + (8u << 20); }

// Loads the predictor shipped next to the library (model/blockparams.f32) unless one is set.
xnyz_status ensure_model(xnyz_ctx* c) {
    if (c->d_model) return XNYZ_OK;
    Dl_info di{};
    std::string path;
    if (const char* env = std::getenv("XNYZ_MODEL")) {
        path = env;
    } else if (dladdr(reinterpret_cast<void*>(&ensure_model), &di) && di.dli_fname) {
        path = di.dli_fname;
        const size_t slash = path.rfind('/');
        path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/model/blockparams.f32";
    }
    std::vector<float> prm(kParamCount);
    FILE* f = path.empty() ? nullptr : std::fopen(path.c_str(), "rb");
    if (!f) return fail(XNYZ_ERR_INVALID_ARG, "no block-parameter model: call xnyz_set_model (looked for " + path + ")");
    const size_t got = std::fread(prm.data(), sizeof(float), prm.size(), f);
    std::fclose(f);
    if (got != prm.size()) return fail(XNYZ_ERR_INVALID_ARG, "block-parameter model file has the wrong size: " + path);
    CUDA_TRY(cudaMalloc(&c->d_model, sizeof(float) * kParamCount));
    CUDA_TRY(cudaMemcpy(c->d_model, prm.data(), sizeof(float) * kParamCount, cudaMemcpyHostToDevice));
    return XNYZ_OK;
}

// Chooses (w, k) per 1024-value block of the repos / SFC-delta values (cp.o_repval) by the
// context's block mode, then the block sizes and offsets (payload bits in Small::ext_bits).
xnyz_status select_block_params(xnyz_ctx* c, const CPlan& cp, uint64_t U, uint64_t nb) {
    cudaStream_t st = c->stream;
    TRY(memset_small(c, offsetof(Small, ext_bits), 3 * sizeof(unsigned long long), 0));
    if (!U) return XNYZ_OK;
    const unsigned long long* rv = at<unsigned long long>(c, cp.o_repval);
    uint8_t* xw = at<uint8_t>(c, cp.o_xw);
    uint8_t* xk = at<uint8_t>(c, cp.o_xk);
    uint32_t* xcost = at<uint32_t>(c, cp.o_xcost);
    if (c->block_mode == XNYZ_BLOCKS_LEARNED) {
        TRY(ensure_model(c));
        float* feats = at<float>(c, cp.o_xfeat);
        float* conf = at<float>(c, cp.o_xconf);
        uint8_t* flags = at<uint8_t>(c, cp.o_xflag);
        {
            Prof pr(c, "block_features", 1, 8.0 * U + 4.0 * kParamFeatures * nb);
            launch_block_features(rv, U, feats, st);
        }
        {
            Prof pr(c, "mlp_forward", 1, 4.0 * kParamFeatures * nb + 10.0 * nb);
            launch_mlp_forward(c->d_model, feats, nb, xw, xk, conf, nullptr, st);
            launch_block_fallback(conf, nb, c->fallback_conf, flags, SMALL_FIELD(c, ext_fallback), st);
        }
        Prof pr(c, "block_search", 1, 8.0 * U);
        launch_block_search(rv, U, flags, xw, xk, nullptr, st);
    } else if (c->block_mode == XNYZ_BLOCKS_EXHAUSTIVE) {
        Prof pr(c, "block_search", 1, 8.0 * U);
        launch_block_search(rv, U, nullptr, xw, xk, nullptr, st);
    } else {
        Prof pr(c, "block_global", 2, 8.0 * U);
        launch_block_global(rv, U, SMALL_FIELD(c, ext_sum), xw, xk, st);
    }
    {
        Prof pr(c, "block_cost", 2, 8.0 * U + 12.0 * nb);
        launch_block_cost(rv, U, xw, xk, xcost, st);
        launch_block_offsets(xcost, nb, at<unsigned long long>(c, cp.o_xoff), SMALL_FIELD(c, ext_bits), st);
    }
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}

// Cell-table input of encode_cells_with_counts (composer/block_compressor_rle.hpp:341-470):
// device cells (int32 xyz) and counts, the global ranges and offset.  Block mode, -rle
// container, one unit per cell, counts carried in the cells' container order.
struct CellInput {
    const int32_t* cells;
    const int32_t* counts;
    int32_t range[3];
    float offset[3];
};

xnyz_status compress_core(xnyz_ctx* c, const float* d_xyz, uint64_t n, const xnyz_params& prm, bool want_order,
                          size_t arena_reserved, CompressOut& R, const CellInput* cin = nullptr) {
    if (prm.quantizer != XNYZ_QUANT_CUBE && prm.quantizer != XNYZ_QUANT_TO && prm.quantizer != XNYZ_QUANT_ADAPTIVE)
        return fail(XNYZ_ERR_INVALID_ARG, "quantizer must be 0 (cube), 1 (truncated octahedron) or 2 (adaptive)");
    if (cin && prm.quantizer == XNYZ_QUANT_ADAPTIVE)
        return fail(XNYZ_ERR_INVALID_ARG, "cell tables take the cube or truncated-octahedron quantizer");
    if (!(prm.l2_bound > 0.0f) || !std::isfinite(prm.l2_bound))
        return fail(XNYZ_ERR_INVALID_ARG, "l2_bound must be a positive finite float");
    if (n == 0) return fail(XNYZ_ERR_INVALID_ARG, "no points (the reference leaves the offset undefined for n = 0)");
    if (n >= (1ull << 31)) return fail(XNYZ_ERR_UNSUPPORTED, "more than 2^31 - 1 points");
    const bool rle = prm.rle != 0, hil = prm.hilbert != 0;
    const bool adaptive = prm.quantizer == XNYZ_QUANT_ADAPTIVE;
    QuantParams q = make_quant(prm.quantizer, prm.l2_bound);
    if (adaptive) q.step_dev = SMALL_FIELD(c, stats.step[0]);  // written by launch_adaptive_steps
    cudaStream_t st = c->stream;

    // ---- 1. bounding box + quantization sweep ----
    HostPhase hp1(c, "c1_stats");
    int32_t* cells_tmp = nullptr;  // the quantization sweep's cells, when the arena holds them
    {
        PointStats init{};
        for (int a = 0; a < 3; ++a) {
            init.minkey[a] = ~0ull;
            init.max_cell[a] = 0;
            init.min_cell[a] = INT32_MAX;
        }
        c->h_small->stats = init;
        c->h_small->err = 0;
        CUDA_TRY(cudaMemcpyAsync(&c->d_small->stats, &c->h_small->stats, sizeof(PointStats), cudaMemcpyHostToDevice, st));
        TRY(memset_small(c, offsetof(Small, err), sizeof(uint32_t), 0));
    }
    if (cin) {
        for (int a = 0; a < 3; ++a) c->h_small->stats.max_cell[a] = INT32_MIN;
        CUDA_TRY(cudaMemcpyAsync(&c->d_small->stats, &c->h_small->stats, sizeof(PointStats), cudaMemcpyHostToDevice, st));
        launch_cells_stats(cin->cells, n, SMALL_FIELD(c, stats), st);
    } else {
        {
            Prof pr(c, "bbox", 1, 12.0 * n);
            launch_bbox(d_xyz, n, SMALL_FIELD(c, stats), st);
        }
        if (adaptive) launch_adaptive_steps(d_xyz, prm.l2_bound, SMALL_FIELD(c, stats), st);
        {
            // the cells go to the space the units fill later, for the block-mode key kernel
            const CPlan cp0 = make_cplan(n, want_order, arena_reserved, c->block_mode != XNYZ_BLOCKS_OFF);
            if (c->arena.cap >= cp0.total) cells_tmp = at<int32_t>(c, cp0.o_patch);  // [o_patch, o_blkunit): 16 n bytes
            Prof pr(c, "quantize_range", 1, 12.0 * n);
            launch_quantize_range(d_xyz, n, q, SMALL_FIELD(c, stats), 1, st, cells_tmp);
        }
    }
    CUDA_TRY(cudaGetLastError());
    TRY(fetch_small(c, offsetof(Small, stats), sizeof(PointStats)));
    PointStats S = c->h_small->stats;
    hp1.end();
    HostPhase hp2(c, "c2_keys_sort_units");
    if (cin) {
        // the reference indexes super-blocks from the given (global) ranges; cells outside
        // them, or below zero other than the z = -1 cells of the truncated octahedron, would
        // wrap its size_t arithmetic
        for (int a = 0; a < 3; ++a)
            if (S.max_cell[a] > cin->range[a] || cin->range[a] < 0)
                return fail(XNYZ_ERR_UNSUPPORTED, "cells outside the given ranges");
        if (S.min_cell[0] < 0 || S.min_cell[1] < 0 || S.min_cell[2] < -1)
            return fail(XNYZ_ERR_UNSUPPORTED, "negative cell coordinates");
        for (int a = 0; a < 3; ++a) {
            S.max_cell[a] = cin->range[a];
            S.offset[a] = cin->offset[a];
        }
        S.mse_max_bits = 0;
        S.mse_sum = 0.0;
    } else {
        if (S.nonfinite) return fail(XNYZ_ERR_UNSUPPORTED, "input contains NaN or infinite coordinates");
        if (S.min_cell[0] < 0 || S.min_cell[1] < 0 || S.min_cell[2] < -1)
            return fail(XNYZ_ERR_UNSUPPORTED, "lattice index outside the int range (coordinates too large for the bound)");
    }
    const int rx = S.max_cell[0], ry = S.max_cell[1], rz = S.max_cell[2];
    const bool defects = S.min_cell[2] < 0;  // truncated-octahedron cells at z = -1
    const int max_range = std::max({rx, ry, rz});
    // cell tables and shared codebooks: always block mode (block_compressor.hpp:314-320)
    const bool shared = c->share_mode != 0;
    if (shared && (rle || cin || c->block_mode != XNYZ_BLOCKS_OFF))
        return fail(XNYZ_ERR_INVALID_ARG, "shared codebooks code the -normal reference container only");
    const bool direct = !cin && !shared && max_range < prm.direct_threshold;

    // ---- 2. key layout ----
    BlockKeyParams bkp{};
    DirectKeyParams dkp{};
    int key_bits = 0;
    const auto& hm = hilbert_machines();
    if (direct) {
        int bits = bitlen(static_cast<uint64_t>(max_range));
        if (bits == 0) bits = 1;
        if (bits > 20) return fail(XNYZ_ERR_UNSUPPORTED, "direct mode with more than 20 bits per axis");
        dkp.bits = bits;
        dkp.hilbert = hil;
        if (defects) {
            dkp.defect_flag = 1ull << (3 * (bits + 1));
            dkp.defect_high = (spread3_host(0x1fffffu) << 2) & ~(dkp.defect_flag - 1);
            key_bits = 3 * (bits + 1) + 1;
        } else {
            key_bits = 3 * bits;
        }
    } else {
        const unsigned __int128 nx = static_cast<uint64_t>(rx) / 128 + 1, ny = static_cast<uint64_t>(ry) / 128 + 1,
                                nz = static_cast<uint64_t>(rz) / 128 + 1;
        const unsigned __int128 cells = nx * ny * nz;
        if (cells > (static_cast<unsigned __int128>(1) << 43))
            return fail(XNYZ_ERR_UNSUPPORTED, "block ids need more than 43 bits");
        const int B = bitlen(static_cast<uint64_t>(cells - 1));
        bkp.nx = static_cast<uint64_t>(nx);
        bkp.ny = static_cast<uint64_t>(ny);
        bkp.hilbert = hil;
        bkp.hstart = hm.fwd_block_start;
        key_bits = B + 21;
        if (defects) {
            // z = -1 wraps to 2^64 - 1 before the division by 64 (block_quantizer.hpp:103):
            // their ids are ((2^58 - 1) / 2) * nx * ny + (cx/2 + cy/2 * nx) modulo 2^64.
            const uint64_t base = ((~0ull >> 6) >> 1) * (static_cast<uint64_t>(nx) * static_cast<uint64_t>(ny));
            const unsigned __int128 top = static_cast<unsigned __int128>(base) + nx * ny;
            if (static_cast<unsigned __int128>(base) < cells || top > (static_cast<unsigned __int128>(1) << 64))
                return fail(XNYZ_ERR_UNSUPPORTED, "z = -1 cells whose block ids interleave the others");
            bkp.defect_base = base;
            bkp.defect_flag = 1ull << (B + 21);
            key_bits = B + 22;
        }
        if (key_bits > 64) return fail(XNYZ_ERR_UNSUPPORTED, "sort keys wider than 64 bits");
    }
    const int passes = static_cast<int>(cdiv(key_bits, 8));

    // ---- 3. arena plan ----
    const bool ext = c->block_mode != XNYZ_BLOCKS_OFF;
    const CPlan cp = make_cplan(n, want_order, arena_reserved, ext);
    const uint64_t tiles = cp.tiles;
    const size_t o_k0 = cp.o_k0, o_k1 = cp.o_k1, o_v0 = cp.o_v0, o_v1 = cp.o_v1, o_rep = cp.o_rep, o_quad = cp.o_quad,
                 o_patch = cp.o_patch, o_blkid = cp.o_blkid, o_blkunit = cp.o_blkunit, o_unitpos = cp.o_unitpos,
                 o_counts = cp.o_counts, o_over_v = cp.o_over_v, o_over_u = cp.o_over_u, o_dblk = cp.o_dblk,
                 o_dcnt = cp.o_dcnt;
    const LB lb_units = cp.lb_units, lb_enc = cp.lb_enc;
    Plan pl;
    pl.total = cp.total;
    (void)tiles;
    TRY(ensure_arena(c, pl.total));

    // ---- 4. keys + digit histograms ----
    SortBufs sb{{at<unsigned long long>(c, o_k0), at<unsigned long long>(c, o_k1)},
                {want_order ? at<uint32_t>(c, o_v0) : nullptr, want_order ? at<uint32_t>(c, o_v1) : nullptr}};
    TRY(memset_small(c, offsetof(Small, sort_hist), sizeof(uint32_t) * 8 * 256, 0));
    CUDA_TRY(cudaMemcpyAsync(c->d_small->hil_fwd, hm.fwd.data(), 256, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemcpyAsync(c->d_small->hil_inv, hm.inv.data(), 256, cudaMemcpyHostToDevice, st));
    {
        Prof pr(c, "keys", 1, 20.0 * n + (want_order ? 4.0 * n : 0.0));
        if (cin)
            launch_keys_cells(cin->cells, n, bkp, c->d_small->hil_fwd, sb.keys[0], sb.vals[0], passes,
                              c->d_small->sort_hist, st);
        else if (direct)
            launch_keys_direct(d_xyz, n, q, SMALL_FIELD(c, stats), dkp, c->d_small->hil_fwd, sb.keys[0], sb.vals[0],
                               passes, c->d_small->sort_hist, st);
        else if (cells_tmp)
            launch_keys_cells(cells_tmp, n, bkp, c->d_small->hil_fwd, sb.keys[0], sb.vals[0], passes,
                              c->d_small->sort_hist, st);
        else
            launch_keys_block(d_xyz, n, q, SMALL_FIELD(c, stats), bkp, c->d_small->hil_fwd, sb.keys[0], sb.vals[0],
                              passes, c->d_small->sort_hist, st);
    }
    int res = 0;
    TRY(radix_sort(c, sb, n, passes, c->d_small->sort_hist, res));
    const unsigned long long* sorted = sb.keys[res];
    if (want_order) R.d_order = sb.vals[res];

    // ---- 5. units ----
    TRY(memset_small(c, offsetof(Small, counters), sizeof(unsigned long long) * 8, 0));
    TRY(memset_small(c, offsetof(Small, hist_rep), sizeof(unsigned long long) * 256, 0));
    TRY(memset_small(c, offsetof(Small, first_rep), sizeof(uint32_t) * 256, 0xff));
    TRY(memset_small(c, offsetof(Small, hist_quad), sizeof(unsigned long long) * 256, 0));
    TRY(memset_small(c, offsetof(Small, first_quad), sizeof(uint32_t) * 256, 0xff));
    TRY(memset_small(c, offsetof(Small, tile_counters), sizeof(uint32_t) * 64, 0));
    TRY(lb_clear(c, lb_units, 3));
    UnitOutputs uo{};
    uo.rep_val = ext ? at<unsigned long long>(c, cp.o_repval) : nullptr;
    uo.rep_sym = at<uint8_t>(c, o_rep);
    uo.quad_sym = at<uint8_t>(c, o_quad);
    uo.patches = at<unsigned long long>(c, o_patch);
    uo.blk_id = at<unsigned long long>(c, o_blkid);
    uo.blk_unit = at<uint32_t>(c, o_blkunit);
    uo.unit_pos = at<uint32_t>(c, o_unitpos);
    uo.hist_rep = c->d_small->hist_rep;
    uo.first_rep = c->d_small->first_rep;
    uo.hist_quad = c->d_small->hist_quad;
    uo.first_quad = c->d_small->first_quad;
    uo.counters = c->d_small->counters;
    {
        Prof pr(c, "units", 1, 8.0 * n);
        if (direct)
            launch_units_direct(sorted, n, rle, dkp, uo, lb_state(c, lb_units), SMALL_FIELD(c, tile_counters[10]),
                                SMALL_FIELD(c, err), st);
        else
            launch_units_block(sorted, n, cin ? 0 : rle, bkp, uo, lb_state(c, lb_units),
                               SMALL_FIELD(c, tile_counters[10]), SMALL_FIELD(c, err), st);
    }
    CUDA_TRY(cudaGetLastError());
    TRY(fetch_small(c, offsetof(Small, counters), sizeof(unsigned long long) * 8));
    const uint64_t U = c->h_small->counters[0], P = c->h_small->counters[1], NB = c->h_small->counters[2];
    const uint64_t psum = c->h_small->counters[3];
    TRY(check_device_errors(c));
    hp2.end();
    HostPhase hp3(c, "c3_stats");

    // ---- 6. count and block statistics ----
    if (rle) {
        TRY(memset_small(c, offsetof(Small, cnt_hist), sizeof(unsigned long long) * kCountDense, 0));
        TRY(memset_small(c, offsetof(Small, cnt_first), sizeof(uint32_t) * kCountDense, 0xff));
        TRY(memset_small(c, offsetof(Small, over_n), sizeof(uint32_t), 0));
        CountStats cs{c->d_small->cnt_hist, c->d_small->cnt_first, at<uint32_t>(c, o_over_v), at<uint32_t>(c, o_over_u),
                      SMALL_FIELD(c, over_n)};
        Prof pr(c, "count_stats", 1, 8.0 * U);
        if (cin) launch_gather_i32(cin->counts, R.d_order, U, at<int32_t>(c, o_counts), st);  // container order
        launch_count_stats(cin ? nullptr : uo.unit_pos, U, n, at<int32_t>(c, o_counts), cs, st);
    }
    if (!direct) {
        TRY(memset_small(c, offsetof(Small, max2), sizeof(unsigned long long) * 2, 0));
        Prof pr(c, "block_deltas", 1, 28.0 * NB);
        launch_block_deltas(uo.blk_id, uo.blk_unit, NB, U, at<unsigned long long>(c, o_dblk),
                            at<unsigned long long>(c, o_dcnt), c->d_small->max2, st);
    }
    // ---- 6b. extended container: block parameters of the repos / SFC-delta stream ----
    const uint64_t ext_nb = ext ? cdiv(U, kParamBlock) : 0;
    if (ext) TRY(select_block_params(c, cp, U, ext_nb));
    CUDA_TRY(cudaGetLastError());
    TRY(fetch_small(c, offsetof(Small, hist_rep),
                    offsetof(Small, tile_counters) - offsetof(Small, hist_rep)));  // hists, counts, maxima
    const Small& H = *c->h_small;
    hp3.end();
    HostPhase hp4(c, "c4_codebooks");

    // ---- 7. codebooks (host replay of the reference's container order) ----
    std::vector<SymbolStat> st_rep, st_quad, st_cnt;
    for (int s = 0; s < 256; ++s) {
        if (H.hist_rep[s]) st_rep.push_back(SymbolStat{static_cast<uint64_t>(s), H.hist_rep[s], H.first_rep[s]});
        if (!direct && H.hist_quad[s])
            st_quad.push_back(SymbolStat{static_cast<uint64_t>(s), H.hist_quad[s], H.first_quad[s]});
    }
    StreamCode code_rep, code_quad;
    if (c->share_mode == 1) {  // fit_profile: codebooks covering every symbol 0..255
        code_rep = build_complete_code(SymType::U64, st_rep, U, 255);
        code_quad = build_complete_code(SymType::U8, st_quad, U, 255);
        c->share_out.clear();
        for (const auto* m : {&code_rep.meta, &code_quad.meta}) {  // serialize_profile layout
            const uint32_t len = static_cast<uint32_t>(m->size());
            for (int b = 0; b < 4; ++b) c->share_out.push_back(static_cast<uint8_t>(len >> (8 * b)));
            c->share_out.insert(c->share_out.end(), m->begin(), m->end());
        }
    } else if (c->share_mode == 2) {  // compress_with_profile: the profile's codebooks
        std::string e;
        if (!loaded_stream_code(SymType::U64, c->share_rep.data(), c->share_rep.size(), st_rep, code_rep, e) ||
            !loaded_stream_code(SymType::U8, c->share_quad.data(), c->share_quad.size(), st_quad, code_quad, e))
            return fail(XNYZ_ERR_INVALID_ARG, "profile: " + e);
    } else {
        if (!ext) code_rep = build_stream_code(SymType::U64, st_rep, U);
        if (!direct) code_quad = build_stream_code(SymType::U8, st_quad, U);
    }
    StreamCode code_cnt;
    std::vector<uint32_t> sparse_val, sparse_bits;
    std::vector<uint8_t> sparse_len;
    std::vector<uint32_t> dense_bits(kCountDense, 0);
    std::vector<uint8_t> dense_len(kCountDense, 0);
    if (rle) {
        for (int v = 0; v < kCountDense; ++v)
            if (H.cnt_hist[v]) st_cnt.push_back(SymbolStat{static_cast<uint64_t>(v), H.cnt_hist[v], H.cnt_first[v]});
        const uint32_t over = H.over_n;
        if (over) {
            std::vector<uint32_t> ov(over), ou(over);
            CUDA_TRY(cudaMemcpyAsync(ov.data(), at<uint32_t>(c, o_over_v), 4ull * over, cudaMemcpyDeviceToHost, st));
            CUDA_TRY(cudaMemcpyAsync(ou.data(), at<uint32_t>(c, o_over_u), 4ull * over, cudaMemcpyDeviceToHost, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            std::unordered_map<uint32_t, std::pair<uint64_t, uint64_t>> agg;  // value -> (count, first unit)
            for (uint32_t i = 0; i < over; ++i) {
                auto& e = agg[ov[i]];
                if (e.first == 0) e.second = ou[i];
                e.first += 1;
                e.second = std::min<uint64_t>(e.second, ou[i]);
            }
            for (auto& kv : agg) st_cnt.push_back(SymbolStat{kv.first, kv.second.first, kv.second.second});
        }
        code_cnt = build_count_code(st_cnt, U);
        if (!code_cnt.exp_golomb) {
            std::vector<std::pair<uint32_t, size_t>> sp;
            for (size_t i = 0; i < code_cnt.symbols.size(); ++i) {
                const uint32_t v = static_cast<uint32_t>(code_cnt.symbols[i]);
                if (v < static_cast<uint32_t>(kCountDense)) {
                    dense_bits[v] = code_cnt.codes[i].bits;
                    dense_len[v] = code_cnt.codes[i].len;
                } else {
                    sp.emplace_back(v, i);
                }
            }
            std::sort(sp.begin(), sp.end());
            for (auto& e : sp) {
                sparse_val.push_back(e.first);
                sparse_bits.push_back(code_cnt.codes[e.second].bits);
                sparse_len.push_back(code_cnt.codes[e.second].len);
            }
        }
    }
    auto to_bytecodes = [](const StreamCode& sc) {
        ByteCodes b{};
        for (size_t i = 0; i < sc.symbols.size(); ++i) {
            const uint64_t s = sc.symbols[i];
            if (s < 256) {
                b.bits[s] = sc.codes[i].bits;
                b.len[s] = sc.codes[i].len;
            }
        }
        return b;
    };
    c->h_small->codes[0] = to_bytecodes(code_rep);
    c->h_small->codes[1] = to_bytecodes(code_quad);
    CUDA_TRY(cudaMemcpyAsync(c->d_small->codes, c->h_small->codes, sizeof(ByteCodes) * 2, cudaMemcpyHostToDevice, st));
    const uint8_t grk = golomb_rice_k(psum, P, false);
    int w_blk = 1, w_cnt = 1;
    if (!direct) {
        w_blk = H.max2[0] == 0 ? 1 : bitlen(H.max2[0]);
        w_cnt = H.max2[1] == 0 ? 1 : bitlen(H.max2[1]);
    }

    hp4.end();
    HostPhase hp5(c, "c5_encode");
    // ---- 8. encoders ----
    // Output sizes: Huffman and bit-pack streams are known exactly; the Golomb-Rice stream is
    // bounded by P*(k+1) + sum(v >> k) <= P*(k+1) + (sum >> k) + P.
    const uint64_t bits_rep = code_rep.encoded_bits, bits_quad = direct ? 0 : code_quad.encoded_bits;
    const uint64_t bits_cnt = rle ? code_cnt.encoded_bits : 0;
    const unsigned __int128 gr_bound =
        ext ? 0 : static_cast<unsigned __int128>(P) * (grk + 2) + (psum >> grk);
    if (gr_bound > (static_cast<unsigned __int128>(1) << 40))
        return fail(XNYZ_ERR_UNSUPPORTED, "Golomb-Rice stream larger than 2^40 bits");
    const uint64_t bits_gr = static_cast<uint64_t>(gr_bound);
    const uint64_t ext_bits = ext ? H.ext_bits : 0;
    auto words_for = [](uint64_t bits) { return cdiv(bits, 32) + 4; };
    Plan pe;
    pe.total = pl.total;
    const size_t o_w_blk = pe.add(4 * words_for(NB * static_cast<uint64_t>(w_blk)));
    const size_t o_w_cnt = pe.add(4 * words_for(NB * static_cast<uint64_t>(w_cnt)));
    const size_t o_w_gr = pe.add(4 * words_for(bits_gr));
    const size_t o_w_rep = pe.add(4 * words_for(bits_rep));
    const size_t o_w_quad = pe.add(4 * words_for(bits_quad));
    const size_t o_w_cn = pe.add(4 * words_for(bits_cnt));
    const size_t o_dense = pe.add(kCountDense * 5);
    const size_t o_sparse = pe.add(sparse_val.size() * 9 + 16);
    const size_t o_w_xp = pe.add(4 * words_for(ext_bits));
    const size_t enc_begin = o_w_blk, enc_end = pe.total;
    if (pe.total > c->arena.cap) {
        // Growing would move the arena; the inputs above live in it.  Plan for the worst
        // case next time and redo this call.
        return fail(XNYZ_ERR_OOM, "__grow__:" + std::to_string(pe.total));
    }
    CUDA_TRY(cudaMemsetAsync(c->arena.base + enc_begin, 0, enc_end - enc_begin, st));
    TRY(memset_small(c, offsetof(Small, totals), sizeof(unsigned long long) * 8, 0));
    TRY(memset_small(c, offsetof(Small, tile_counters), sizeof(uint32_t) * 64, 0));
    TRY(lb_clear(c, lb_enc, 4));
    const LookBackState lbs = lb_state(c, lb_enc);
    auto chan = [&](int ch) {
        return LookBackState{lbs.flag + ch * lb_enc.tiles, lbs.agg + ch * lb_enc.tiles, lbs.inc + ch * lb_enc.tiles};
    };
    if (!direct) {
        Prof pr(c, "bitpack", 2, 16.0 * NB + (w_blk + w_cnt) * NB / 8.0);
        launch_bitpack(at<unsigned long long>(c, o_dblk), NB, w_blk, at<uint32_t>(c, o_w_blk), st);
        launch_bitpack(at<unsigned long long>(c, o_dcnt), NB, w_cnt, at<uint32_t>(c, o_w_cnt), st);
    }
    // The four entropy coders are independent: one side stream each.
    uint32_t* dbits = at<uint32_t>(c, o_dense);
    uint8_t* dlen = reinterpret_cast<uint8_t*>(dbits + kCountDense);
    uint32_t* sval = at<uint32_t>(c, o_sparse);
    uint32_t* sbits = sval + sparse_val.size();
    uint8_t* slen = reinterpret_cast<uint8_t*>(sbits + sparse_val.size());
    if (rle) {
        CUDA_TRY(cudaMemcpyAsync(dbits, dense_bits.data(), 4 * kCountDense, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(dlen, dense_len.data(), kCountDense, cudaMemcpyHostToDevice, st));
        if (!sparse_val.empty()) {
            CUDA_TRY(cudaMemcpyAsync(sval, sparse_val.data(), 4 * sparse_val.size(), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(sbits, sparse_bits.data(), 4 * sparse_val.size(), cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaMemcpyAsync(slen, sparse_len.data(), sparse_val.size(), cudaMemcpyHostToDevice, st));
        }
    }
    TRY(fork_sides(c));
    if (ext && U) {
        Prof pr(c, "encode_blocks", 1, 8.0 * U + ext_bits / 8.0, side(c, 0));
        launch_block_encode(at<unsigned long long>(c, cp.o_repval), U, at<uint8_t>(c, cp.o_xw), at<uint8_t>(c, cp.o_xk),
                            at<unsigned long long>(c, cp.o_xoff), at<uint32_t>(c, o_w_xp), side(c, 0));
    }
    if (P && !ext) {
        Prof pr(c, "encode_golomb_rice", 1, 8.0 * P + bits_gr / 8.0, side(c, 0));
        launch_gr_encode(uo.patches, P, grk, at<uint32_t>(c, o_w_gr), 32 * words_for(bits_gr), chan(0),
                         SMALL_FIELD(c, tile_counters[0]), SMALL_FIELD(c, totals[0]), SMALL_FIELD(c, err), side(c, 0));
    }
    // A code whose codewords all have one length (quads at fine bounds: eight 3-bit codes;
    // most -rle count streams: two 1-bit codes) places symbol i at bits [i L, (i + 1) L).
    const int fl_rep = fixed_code_len(c->h_small->codes[0].len, 256);
    const int fl_quad = fixed_code_len(c->h_small->codes[1].len, 256);
    const int fl_cnt = (rle && !code_cnt.exp_golomb && sparse_val.empty()) ? fixed_code_len(dense_len.data(), kCountDense) : 0;
    if (!ext && !code_rep.exp_golomb) {
        Prof pr(c, "encode_huffman", 1, 1.0 * U + bits_rep / 8.0, side(c, 1));
        if (fl_rep)
            launch_fixed_encode_u8(uo.rep_sym, U, c->d_small->codes[0].bits, fl_rep, at<uint32_t>(c, o_w_rep),
                                   SMALL_FIELD(c, totals[1]), side(c, 1));
        else
            launch_huff_encode_u8(uo.rep_sym, U, &c->d_small->codes[0], at<uint32_t>(c, o_w_rep), 32 * words_for(bits_rep),
                                  chan(1), SMALL_FIELD(c, tile_counters[1]), SMALL_FIELD(c, totals[1]), SMALL_FIELD(c, err),
                                  side(c, 1));
    }
    if (!direct) {
        Prof pr(c, "encode_huffman", 1, 1.0 * U + bits_quad / 8.0, side(c, 2));
        if (fl_quad)
            launch_fixed_encode_u8(uo.quad_sym, U, c->d_small->codes[1].bits, fl_quad, at<uint32_t>(c, o_w_quad),
                                   SMALL_FIELD(c, totals[2]), side(c, 2));
        else
            launch_huff_encode_u8(uo.quad_sym, U, &c->d_small->codes[1], at<uint32_t>(c, o_w_quad),
                                  32 * words_for(bits_quad), chan(2), SMALL_FIELD(c, tile_counters[2]),
                                  SMALL_FIELD(c, totals[2]), SMALL_FIELD(c, err), side(c, 2));
    }
    if (rle && fl_cnt) {
        Prof pr(c, "encode_counts", 1, 4.0 * U + bits_cnt / 8.0, side(c, 3));
        launch_fixed_encode_i32(at<int32_t>(c, o_counts), U, dbits, fl_cnt, at<uint32_t>(c, o_w_cn),
                                SMALL_FIELD(c, totals[3]), side(c, 3));
    } else if (rle) {
        Prof pr(c, "encode_counts", 1, 4.0 * U + bits_cnt / 8.0, side(c, 3));
        launch_count_encode(at<int32_t>(c, o_counts), U, code_cnt.exp_golomb ? code_cnt.eg_k : -1, dbits, dlen, sval,
                            sbits, slen, static_cast<uint32_t>(sparse_val.size()), at<uint32_t>(c, o_w_cn),
                            32 * words_for(bits_cnt), chan(3), SMALL_FIELD(c, tile_counters[3]),
                            SMALL_FIELD(c, totals[3]), SMALL_FIELD(c, err), side(c, 3));
    }
    CUDA_TRY(cudaGetLastError());
    TRY(join_sides(c));
    TRY(fetch_small(c, offsetof(Small, err), offsetof(Small, codewords) - offsetof(Small, err)));  // err .. totals
    TRY(device_errors(c));
    const uint64_t gr_bits = c->h_small->totals[0];
    if (!ext && !code_rep.exp_golomb && c->h_small->totals[1] != bits_rep)
        return fail(XNYZ_ERR_CUDA, "Huffman encoder size mismatch (repos)");
    if (!direct && c->h_small->totals[2] != bits_quad) return fail(XNYZ_ERR_CUDA, "Huffman encoder size mismatch (quads)");
    if (rle && c->h_small->totals[3] != bits_cnt) return fail(XNYZ_ERR_CUDA, "count encoder size mismatch");

    hp5.end();
    HostPhase hp6(c, "c6_container");
    // ---- 9. container (Appendix: block_compressor.hpp:56-215, block_compressor_rle.hpp:125-314) ----
    Container& K = R.cont;
    if (ext) K.pod<uint64_t>(kExtMagic);
    K.pod<uint64_t>(U);
    if (adaptive) {  // params: the adaptive quantizer's three steps (block_compressor.hpp:63-66)
        K.pod<uint64_t>(3);
        for (int a = 0; a < 3; ++a) K.pod<float>(S.step[a]);
    } else {
        K.pod<uint64_t>(0);  // the cube and truncated-octahedron quantizers have none
    }
    K.pod<int32_t>(rx);
    K.pod<int32_t>(ry);
    K.pod<int32_t>(rz);
    K.pod<uint8_t>(hil ? 1 : 0);
    K.pod<uint8_t>(direct ? 1 : 0);
    const std::vector<uint8_t> gr_meta = P ? le5(static_cast<uint32_t>(P), grk) : std::vector<uint8_t>{};
    // the repos / SFC-delta stream: GR(patches) + Huffman(PFor symbols), or the block stream
    auto rep_streams = [&]() {
        if (ext) {
            std::vector<uint8_t> meta(16);
            std::memcpy(meta.data(), &U, 8);
            std::memcpy(meta.data() + 8, &ext_bits, 8);
            const size_t pad = (8 - (2 * ext_nb) % 8) % 8;
            K.stream_parts(meta, {{at<uint8_t>(c, cp.o_xw), ext_nb},
                                  {at<uint8_t>(c, cp.o_xk), ext_nb},
                                  {nullptr, pad},
                                  {at<unsigned long long>(c, cp.o_xoff), 8 * ext_nb},
                                  {at<uint32_t>(c, o_w_xp), cdiv(ext_bits, 8)}});
            K.stream({}, nullptr, 0);
        } else {
            K.stream(gr_meta, at<uint32_t>(c, o_w_gr), P ? cdiv(gr_bits, 8) : 0);
            K.stream(code_rep.meta, at<uint32_t>(c, o_w_rep), cdiv(bits_rep, 8));
        }
    };
    if (direct) {
        rep_streams();
    } else {
        K.stream(le5(static_cast<uint32_t>(NB), static_cast<uint8_t>(w_blk)), at<uint32_t>(c, o_w_blk),
                 cdiv(NB * static_cast<uint64_t>(w_blk), 8));
        K.stream(le5(static_cast<uint32_t>(NB), static_cast<uint8_t>(w_cnt)), at<uint32_t>(c, o_w_cnt),
                 cdiv(NB * static_cast<uint64_t>(w_cnt), 8));
        rep_streams();
        K.stream({}, nullptr, 0);  // quad patches: quad deltas are < 8, never patched
        K.stream(code_quad.meta, at<uint32_t>(c, o_w_quad), cdiv(bits_quad, 8));
    }
    if (rle) K.stream(code_cnt.meta, at<uint32_t>(c, o_w_cn), cdiv(bits_cnt, 8));
    K.pod<float>(S.offset[0]);
    K.pod<float>(S.offset[1]);
    K.pod<float>(S.offset[2]);

    xnyz_compress_info& I = R.info;
    I.num_points = n;
    I.num_units = U;
    I.num_blocks = direct ? 0 : NB;
    I.num_patches = P;
    I.container_bytes = K.size;
    I.range[0] = rx;
    I.range[1] = ry;
    I.range[2] = rz;
    I.is_direct = direct;
    I.counts_exp_golomb = rle && code_cnt.exp_golomb;
    float emax;
    std::memcpy(&emax, &S.mse_max_bits, 4);
    I.max_l2_error = std::sqrt(static_cast<double>(emax));
    I.mse = S.mse_sum / static_cast<double>(n);
    c->last_blocks = xnyz_block_info{};
    c->last_repval = ext ? at<unsigned long long>(c, cp.o_repval) : nullptr;
    c->last_repval_n = ext ? U : 0;
    if (ext) {
        c->last_blocks.values = U;
        c->last_blocks.blocks = ext_nb;
        c->last_blocks.payload_bits = ext_bits;
        c->last_blocks.fallback_blocks = H.ext_fallback;
        c->last_blocks.mode = c->block_mode;
    }
    return XNYZ_OK;
}

// Runs compress_core, growing the arena and retrying once when the encoders need more.
xnyz_status compress_run(xnyz_ctx* c, const float* d_xyz, uint64_t n, const xnyz_params& p, bool want_order,
                         size_t reserved, CompressOut& R, const CellInput* cin = nullptr) {
    xnyz_status s = compress_core(c, d_xyz, n, p, want_order, reserved, R, cin);
    if (s == XNYZ_ERR_OOM && g_last_error.rfind("__grow__:", 0) == 0) {
        const size_t need = std::stoull(g_last_error.substr(9));
        // Input points may live in the arena's reserved prefix: keep them.
        if (reserved) {
            char* old = c->arena.base;
            char* fresh = nullptr;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            CUDA_TRY(cudaMalloc(&fresh, align_up(need + need / 8, 1 << 20)));
            CUDA_TRY(cudaMemcpyAsync(fresh, old, reserved, cudaMemcpyDeviceToDevice, c->stream));
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            cudaFree(old);
            const ptrdiff_t shift = fresh - old;
            c->arena.base = fresh;
            c->arena.cap = align_up(need + need / 8, 1 << 20);
            d_xyz = reinterpret_cast<const float*>(reinterpret_cast<const char*>(d_xyz) + shift);
        } else {
            TRY(ensure_arena(c, need));
        }
        R = CompressOut{};
        s = compress_core(c, d_xyz, n, p, want_order, reserved, R, cin);
    }
    return s;
}

// ---------------------------------------------------------------- header parse -----------
struct StreamRef {
    uint64_t meta_off = 0, meta_len = 0, data_off = 0, data_len = 0;
    std::vector<uint8_t> meta;
};
struct Header {
    bool ext = false;  // extended container (block-coded repos / SFC-delta stream)
    uint64_t units = 0;
    int32_t rx = 0, ry = 0, rz = 0;
    bool hilbert = false, direct = false;
    std::vector<StreamRef> streams;
    std::vector<float> params;  // quantizer parameters (adaptive: the three steps)
    float off[3] = {0, 0, 0};
};

// Reads the container layout (block_decompressor.hpp:40-176, block_decompressor_rle.hpp:41-202)
// through `rd(offset, bytes, dst)`.
template <typename Read>
xnyz_status parse_header(Read rd, uint64_t len, bool rle, Header& h) {
    uint64_t p = 0;
    auto get = [&](void* dst, uint64_t bytes) -> bool {
        if (bytes > len || p > len - bytes) return false;
        if (!rd(p, bytes, dst)) return false;
        p += bytes;
        return true;
    };
    uint64_t np = 0;
    uint8_t hb = 0, db = 0;
    if (!get(&h.units, 8)) return fail(XNYZ_ERR_BAD_STREAM, "truncated container header");
    if (h.units == kExtMagic) {
        h.ext = true;
        if (!get(&h.units, 8)) return fail(XNYZ_ERR_BAD_STREAM, "truncated container header");
    }
    if (!get(&np, 8)) return fail(XNYZ_ERR_BAD_STREAM, "truncated container header");
    if (np > (len - p) / 4) return fail(XNYZ_ERR_BAD_STREAM, "bad parameter count");
    h.params.assign(np < 3 ? np : 3, 0.0f);  // only the adaptive quantizer reads them (three)
    if (!h.params.empty() && !get(h.params.data(), 4 * h.params.size()))
        return fail(XNYZ_ERR_BAD_STREAM, "truncated container header");
    p += 4 * (np - h.params.size());
    if (!get(&h.rx, 4) || !get(&h.ry, 4) || !get(&h.rz, 4) || !get(&hb, 1) || !get(&db, 1))
        return fail(XNYZ_ERR_BAD_STREAM, "truncated container header");
    h.hilbert = hb != 0;
    h.direct = db != 0;
    const int ns = (h.direct ? 2 : 6) + (rle ? 1 : 0);
    for (int i = 0; i < ns; ++i) {
        StreamRef s;
        if (!get(&s.data_len, 8) || !get(&s.meta_len, 8)) return fail(XNYZ_ERR_BAD_STREAM, "truncated stream header");
        if (s.meta_len > len - p) return fail(XNYZ_ERR_BAD_STREAM, "truncated stream meta");
        s.meta_off = p;
        s.meta.resize(s.meta_len);
        if (s.meta_len && !get(s.meta.data(), s.meta_len)) return fail(XNYZ_ERR_BAD_STREAM, "truncated stream meta");
        if (s.data_len > len - p) return fail(XNYZ_ERR_BAD_STREAM, "truncated stream data");
        s.data_off = p;
        p += s.data_len;
        h.streams.push_back(std::move(s));
    }
    if (!get(h.off, 12)) return fail(XNYZ_ERR_BAD_STREAM, "truncated offset");
    return XNYZ_OK;
}

uint32_t le32(const std::vector<uint8_t>& m) {
    return static_cast<uint32_t>(m[0]) | (static_cast<uint32_t>(m[1]) << 8) | (static_cast<uint32_t>(m[2]) << 16) |
           (static_cast<uint32_t>(m[3]) << 24);
}

// Host-built decode tables of one Huffman stream.
struct HuffTables {
    int root_bits = 1;
    int max_len = 0;
    std::vector<uint32_t> root, tree;
    std::vector<unsigned long long> symvals;
    bool direct_values = false;  // table payloads are the symbol values (all below 2^24)
};

xnyz_status build_huff_tables(const ParsedMeta& pm, HuffTables& t) {
    t = HuffTables{};
    for (const auto& c : pm.codes) t.max_len = std::max<int>(t.max_len, c.len);
    if (t.max_len > 32) return fail(XNYZ_ERR_UNSUPPORTED, "Huffman codes longer than 32 bits");
    if (pm.symbols.size() >= (1u << 24)) return fail(XNYZ_ERR_UNSUPPORTED, "Huffman alphabet too large");
    t.root_bits = std::max(1, std::min(t.max_len, 11));
    const int rb = t.root_bits;
    t.root.assign(1u << rb, 0u);
    t.symvals.assign(pm.symbols.begin(), pm.symbols.end());
    t.direct_values = true;
    for (unsigned long long v : t.symvals)
        if (v >= (1ull << 24)) t.direct_values = false;
    auto payload = [&](size_t oi) {
        return t.direct_values ? static_cast<uint32_t>(t.symvals[oi]) : static_cast<uint32_t>(oi);
    };
    // Longer codes first so that a shorter code sharing a prefix wins, as the reference's
    // bit-by-bit matcher stops at the first (shortest) match.
    std::vector<size_t> order(pm.codes.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return pm.codes[a].len > pm.codes[b].len; });
    for (size_t oi : order) {
        const CodeEntry& ce = pm.codes[oi];
        const int len = ce.len;
        if (len == 0) continue;
        const uint32_t bits = len >= 32 ? ce.bits : (ce.bits & ((1u << len) - 1u));
        if (len <= rb) {
            const uint32_t first = bits << (rb - len), span = 1u << (rb - len);
            for (uint32_t k = 0; k < span; ++k) t.root[first + k] = (static_cast<uint32_t>(len) << 24) | payload(oi);
        } else {
            const uint32_t top = bits >> (len - rb);
            uint32_t& e = t.root[top];
            uint32_t node;
            if (e == 0u) {
                node = static_cast<uint32_t>(t.tree.size() / 2);
                t.tree.push_back(0xffffffffu);
                t.tree.push_back(0xffffffffu);
                e = 0x80000000u | node;
            } else if (e & 0x80000000u) {
                node = e & 0x7fffffffu;
            } else {
                continue;  // shadowed by a shorter code
            }
            bool shadowed = false;
            for (int i = len - rb - 1; i >= 1; --i) {
                const uint32_t b = (bits >> i) & 1u;
                uint32_t& ch = t.tree[2 * node + b];
                if (ch == 0xffffffffu) {
                    const uint32_t nn = static_cast<uint32_t>(t.tree.size() / 2);
                    t.tree.push_back(0xffffffffu);
                    t.tree.push_back(0xffffffffu);
                    t.tree[2 * node + b] = nn;
                    node = nn;
                } else if (ch & 0x80000000u) {
                    shadowed = true;
                    break;
                } else {
                    node = ch;
                }
            }
            if (shadowed) continue;
            uint32_t& leaf = t.tree[2 * node + (bits & 1u)];
            if (leaf == 0xffffffffu) leaf = 0x80000000u | payload(oi);
        }
    }
    if (t.tree.empty()) t.tree.assign(2, 0xffffffffu);
    return XNYZ_OK;
}

struct DecodeJob {
    int kind = 0;
    const uint32_t* words = nullptr;
    uint64_t base_bits = 0, total_bits = 0, nsym = 0;
    int width = 1;
    void* out = nullptr;
    DecodeTable table{};
    int L = 1;
    int slot = 0;
    bool fill = false;
    uint64_t fill_value = 0;
    int fixed_len = 0;  // Huffman: every codeword has this length (decoded without entry tables)
};

// cells_out: decompress_to_cells (block_decompressor_rle.hpp:230-335): *d_out receives the
// units' lattice cells (int32 xyz, container order, not expanded) and *cells_out the decoded
// counts; otherwise *d_out receives the points.
xnyz_status decompress_core(xnyz_ctx* c, const uint8_t* d_cont, uint64_t len, const Header& h, int quantizer,
                            float l2, bool rle, size_t reserved, float** d_out, uint64_t* n_out,
                            int32_t** cells_out = nullptr) {
    cudaStream_t st = c->stream;
    // BlockDecompressorRLE picks the truncated octahedron or else the cube quantizer
    // (block_decompressor_rle.hpp:189-196): adaptive -rle containers recover as cube cells.
    const int qrec = (rle && quantizer == XNYZ_QUANT_ADAPTIVE) ? XNYZ_QUANT_CUBE : quantizer;
    QuantParams q = make_quant(qrec, l2);
    if (qrec == XNYZ_QUANT_ADAPTIVE) {
        if (h.params.size() < 3) return fail(XNYZ_ERR_BAD_STREAM, "adaptive container without its three steps");
        for (int a = 0; a < 3; ++a) q.step[a] = h.params[a];
    }
    const uint64_t U = h.units;
    if (U >= (1ull << 31)) return fail(XNYZ_ERR_UNSUPPORTED, "more than 2^31 - 1 cells");
    const auto& hm = hilbert_machines();
    auto words_of = [&](const StreamRef& s, uint64_t& base) {
        base = (s.data_off & 3u) * 8u;
        return reinterpret_cast<const uint32_t*>(d_cont + (s.data_off & ~static_cast<uint64_t>(3)));
    };

    HostPhase hd1(c, "d1_metas_tables");
    // ---- stream metas ----
    const int i_gr = h.direct ? 0 : 2, i_sym = h.direct ? 1 : 3;
    const StreamRef& s_gr = h.streams[i_gr];
    const StreamRef& s_sym = h.streams[i_sym];
    uint64_t P = 0;
    uint8_t grk = 0;
    // extended container: the block-coded stream in the Golomb-Rice slot, the symbol slot empty
    uint64_t x_nb = 0, x_bits = 0;
    if (h.ext) {
        if (s_gr.meta.size() != 16 || !s_sym.meta.empty() || s_sym.data_len)
            return fail(XNYZ_ERR_BAD_STREAM, "malformed block-coded stream");
        uint64_t nv = 0;
        std::memcpy(&nv, s_gr.meta.data(), 8);
        std::memcpy(&x_bits, s_gr.meta.data() + 8, 8);
        if (nv != U) return fail(XNYZ_ERR_BAD_STREAM, "block-coded stream and point count disagree");
        x_nb = cdiv(U, kParamBlock);
        const uint64_t pad = (8 - (2 * x_nb) % 8) % 8;
        if (x_bits > (1ull << 50) || s_gr.data_len != 2 * x_nb + pad + 8 * x_nb + cdiv(x_bits, 8))
            return fail(XNYZ_ERR_BAD_STREAM, "block-coded stream has the wrong size");
    } else if (!(s_gr.meta.empty() && s_gr.data_len == 0)) {
        if (s_gr.meta.size() != 5) return fail(XNYZ_ERR_BAD_STREAM, "Invalid meta size in Golomb-Rice packed data");
        P = le32(s_gr.meta);
        grk = s_gr.meta[4];
        if (P && grk >= 63) return fail(XNYZ_ERR_BAD_STREAM, "Invalid k_param in Golomb-Rice packed data meta");
    }
    std::string perr;
    ParsedMeta pm_sym, pm_quad, pm_cnt;
    if (!h.ext && !parse_meta(SymType::U64, s_sym.meta.data(), s_sym.meta.size(), pm_sym, perr))
        return fail(XNYZ_ERR_BAD_STREAM, perr);
    uint64_t NB = 0;
    int w_blk = 0, w_cnt = 0;
    if (!h.direct) {
        const StreamRef& sb = h.streams[0];
        const StreamRef& sc = h.streams[1];
        if (sb.meta.size() != 5 || sc.meta.size() != 5) return fail(XNYZ_ERR_BAD_STREAM, "Invalid meta size in bitpacked data");
        NB = le32(sb.meta);
        w_blk = sb.meta[4];
        w_cnt = sc.meta[4];
        if (le32(sc.meta) != NB) return fail(XNYZ_ERR_BAD_STREAM, "block and count streams disagree");
        if (w_blk > 64 || w_cnt > 64) return fail(XNYZ_ERR_UNSUPPORTED, "bit width above 64");
        if (NB * static_cast<uint64_t>(w_blk) > sb.data_len * 8 || NB * static_cast<uint64_t>(w_cnt) > sc.data_len * 8)
            return fail(XNYZ_ERR_BAD_STREAM, "truncated bit-packed stream");
        const StreamRef& sqp = h.streams[4];
        if (!(sqp.meta.empty() && sqp.data_len == 0)) {
            if (sqp.meta.size() != 5) return fail(XNYZ_ERR_BAD_STREAM, "Invalid meta size in Golomb-Rice packed data");
            if (le32(sqp.meta) != 0) return fail(XNYZ_ERR_UNSUPPORTED, "patched quad deltas (never produced by the encoder)");
        }
        if (!parse_meta(SymType::U8, h.streams[5].meta.data(), h.streams[5].meta.size(), pm_quad, perr))
            return fail(XNYZ_ERR_BAD_STREAM, perr);
        if (pm_quad.exp_golomb) return fail(XNYZ_ERR_UNSUPPORTED, "exp-Golomb quad stream");
    }
    if (pm_sym.exp_golomb) return fail(XNYZ_ERR_UNSUPPORTED, "exp-Golomb repos stream");
    for (uint64_t s : pm_sym.symbols)
        if (s > 255) return fail(XNYZ_ERR_UNSUPPORTED, "repos symbols above 255 (never produced by the encoder)");
    const StreamRef* s_cnt = rle ? &h.streams.back() : nullptr;
    if (rle && !parse_meta(SymType::I32, s_cnt->meta.data(), s_cnt->meta.size(), pm_cnt, perr))
        return fail(XNYZ_ERR_BAD_STREAM, perr);

    // ---- arena plan ----
    Plan pl;
    pl.total = reserved;
    const size_t o_blk = pl.add(8 * NB + 8);
    const size_t o_patch = pl.add(8 * P + 8);
    const size_t o_rep = pl.add(U + 8), o_quad = pl.add(U + 8), o_isst = pl.add(U + 8), o_stb = pl.add(4 * U + 8);
    const size_t o_counts = pl.add(4 * U + 8);
    const size_t o_xw = h.ext ? pl.add(x_nb) : 0, o_xk = h.ext ? pl.add(x_nb) : 0, o_xoff = h.ext ? pl.add(8 * x_nb) : 0,
                 o_xpay = h.ext ? pl.add(4 * (cdiv(x_bits, 32) + 2)) : 0, o_rv = h.ext ? pl.add(8 * U + 8) : 0;
    const LB lb_scan = plan_lb(pl, cdiv(std::max<uint64_t>(NB, 1), kScanTile), 4);
    struct TabOff {
        size_t root, tree, sym;
    };
    HuffTables ht_sym, ht_quad, ht_cnt;
    if (!h.ext) TRY(build_huff_tables(pm_sym, ht_sym));
    if (!h.direct) TRY(build_huff_tables(pm_quad, ht_quad));
    if (rle && !pm_cnt.exp_golomb) TRY(build_huff_tables(pm_cnt, ht_cnt));
    auto plan_tab = [&](const HuffTables& t) {
        return TabOff{pl.add(4 * t.root.size()), pl.add(4 * t.tree.size()), pl.add(8 * t.symvals.size() + 8)};
    };
    const TabOff to_sym = plan_tab(ht_sym), to_quad = plan_tab(ht_quad), to_cnt = plan_tab(ht_cnt);
    // decode look-back state per stream (up to 4 streams)
    auto dec_tiles = [](uint64_t bits) { return cdiv(cdiv(std::max<uint64_t>(bits, 1), kDecodeSubBits), kDecodeBlockSubs); };
    const uint64_t dtiles = std::max({dec_tiles(s_gr.data_len * 8), dec_tiles(s_sym.data_len * 8),
                                      h.direct ? 1 : dec_tiles(h.streams[5].data_len * 8),
                                      rle ? dec_tiles(s_cnt->data_len * 8) : 1});
    size_t o_dflag[4], o_dagg[4], o_dinc[4];
    for (int i = 0; i < 4; ++i) {
        o_dflag[i] = pl.add(4 * dtiles);
        o_dagg[i] = pl.add(8 * dtiles * kDecodeMaxL);
        o_dinc[i] = pl.add(16 * dtiles);
    }
    const uint64_t rtiles = cdiv(std::max<uint64_t>(U, 1), kScanTile);
    const size_t o_rflag = pl.add(4 * rtiles * 5), o_ragg = pl.add(16 * rtiles * 5), o_rinc = pl.add(16 * rtiles * 5);
    if (pl.total > c->arena.cap) return fail(XNYZ_ERR_OOM, "__grow__:" + std::to_string(pl.total));

    TRY(memset_small(c, offsetof(Small, err), sizeof(uint32_t), 0));
    TRY(memset_small(c, offsetof(Small, tile_counters), sizeof(uint32_t) * 64, 0));
    TRY(memset_small(c, offsetof(Small, fallback), sizeof(uint32_t) * 8 * 2, 0));  // fallback + maxrun
    TRY(memset_small(c, offsetof(Small, codewords), sizeof(unsigned long long) * 8, 0));
    CUDA_TRY(cudaMemcpyAsync(c->d_small->hil_inv, hm.inv.data(), 256, cudaMemcpyHostToDevice, st));
    auto upload = [&](const HuffTables& t, const TabOff& o) -> xnyz_status {
        if (!t.root.empty())
            CUDA_TRY(cudaMemcpyAsync(at<uint32_t>(c, o.root), t.root.data(), 4 * t.root.size(), cudaMemcpyHostToDevice, st));
        if (!t.tree.empty())
            CUDA_TRY(cudaMemcpyAsync(at<uint32_t>(c, o.tree), t.tree.data(), 4 * t.tree.size(), cudaMemcpyHostToDevice, st));
        if (!t.symvals.empty())
            CUDA_TRY(cudaMemcpyAsync(at<unsigned long long>(c, o.sym), t.symvals.data(), 8 * t.symvals.size(),
                                     cudaMemcpyHostToDevice, st));
        return XNYZ_OK;
    };
    TRY(upload(ht_sym, to_sym));
    TRY(upload(ht_quad, to_quad));
    TRY(upload(ht_cnt, to_cnt));

    hd1.end();
    HostPhase hd2(c, "d2_launch");
    // The entropy-coded streams decode on the side streams while the block streams are
    // unpacked and scanned on the context's stream.
    TRY(fork_sides(c));
    // ---- block streams: bit-unpack + prefix sums ----
    if (!h.direct && NB) {
        uint64_t b0, b1;
        const uint32_t* w0 = words_of(h.streams[0], b0);
        const uint32_t* w1 = words_of(h.streams[1], b1);
        Prof pr(c, "block_streams", 1, (w_blk + w_cnt) * NB / 8.0 + 8.0 * NB + 5.0 * std::min(NB, U));
        TRY(lb_clear(c, lb_scan, 2));
        CUDA_TRY(cudaMemsetAsync(at<uint8_t>(c, o_isst), 0, U + 8, st));
        launch_block_streams(w0, b0, w_blk, w1, b1, w_cnt, NB, U, at<unsigned long long>(c, o_blk),
                             at<uint8_t>(c, o_isst), at<uint32_t>(c, o_stb), lb_state(c, lb_scan),
                             SMALL_FIELD(c, tile_counters[20]), SMALL_FIELD(c, count_total), SMALL_FIELD(c, err), st);
    }

    // ---- entropy-coded streams ----
    std::vector<DecodeJob> jobs;
    auto huff_job = [&](const StreamRef& s, const ParsedMeta& pm, const HuffTables& t, const TabOff& o, int width,
                        void* out, int slot) -> xnyz_status {
        DecodeJob j;
        j.kind = kCodeHuffman;
        j.words = words_of(s, j.base_bits);
        j.total_bits = s.data_len * 8;
        j.nsym = U;
        j.width = width;
        j.out = out;
        j.slot = slot;
        if (U == 0) return XNYZ_OK;
        if (pm.distinct == 0) return fail(XNYZ_ERR_BAD_STREAM, "empty Huffman table");
        if (pm.distinct == 1) {  // decode(): one code -> every symbol is that symbol
            j.fill = true;
            j.fill_value = pm.symbols[0];
        }
        j.table.root = at<uint32_t>(c, o.root);
        j.table.tree = at<uint32_t>(c, o.tree);
        j.table.symvals = t.direct_values ? nullptr : at<unsigned long long>(c, o.sym);
        j.table.root_bits = t.root_bits;
        j.L = std::max(1, t.max_len);
        bool same = !pm.codes.empty();
        for (const auto& ce : pm.codes) same = same && ce.len == t.max_len;
        if (same && t.max_len == t.root_bits) j.fixed_len = t.max_len;
        jobs.push_back(j);
        return XNYZ_OK;
    };
    if (P) {
        DecodeJob j;
        j.kind = kCodeGolombRice;
        j.words = words_of(s_gr, j.base_bits);
        j.total_bits = s_gr.data_len * 8;
        j.nsym = P;
        j.width = 8;
        j.out = at<unsigned long long>(c, o_patch);
        j.table.param = grk;
        j.slot = 0;
        j.L = -1;  // from the longest one-run
        jobs.push_back(j);
    }
    if (!h.ext) TRY(huff_job(s_sym, pm_sym, ht_sym, to_sym, 1, at<uint8_t>(c, o_rep), 1));
    if (!h.direct) TRY(huff_job(h.streams[5], pm_quad, ht_quad, to_quad, 1, at<uint8_t>(c, o_quad), 2));
    if (rle) {
        if (pm_cnt.exp_golomb) {
            DecodeJob j;
            j.kind = kCodeExpGolomb;
            j.words = words_of(*s_cnt, j.base_bits);
            j.total_bits = s_cnt->data_len * 8;
            j.nsym = U;
            j.width = 4;
            j.out = at<int32_t>(c, o_counts);
            j.table.param = pm_cnt.eg_k;
            j.table.zigzag = 1;
            j.L = kDecodeMaxL;
            j.slot = 3;
            if (U) jobs.push_back(j);
        } else {
            TRY(huff_job(*s_cnt, pm_cnt, ht_cnt, to_cnt, 4, at<int32_t>(c, o_counts), 3));
        }
    }
    if (h.ext && U) {
        // block-coded stream: copy its parts to aligned buffers, then decode every block
        cudaStream_t xs = side(c, 0);
        const uint8_t* src = d_cont + s_gr.data_off;
        const uint64_t pad = (8 - (2 * x_nb) % 8) % 8;
        CUDA_TRY(cudaMemcpyAsync(at<uint8_t>(c, o_xw), src, x_nb, cudaMemcpyDeviceToDevice, xs));
        CUDA_TRY(cudaMemcpyAsync(at<uint8_t>(c, o_xk), src + x_nb, x_nb, cudaMemcpyDeviceToDevice, xs));
        CUDA_TRY(cudaMemcpyAsync(at<uint8_t>(c, o_xoff), src + 2 * x_nb + pad, 8 * x_nb, cudaMemcpyDeviceToDevice, xs));
        CUDA_TRY(cudaMemsetAsync(at<uint8_t>(c, o_xpay), 0, 4 * (cdiv(x_bits, 32) + 2), xs));
        CUDA_TRY(cudaMemcpyAsync(at<uint8_t>(c, o_xpay), src + 2 * x_nb + pad + 8 * x_nb, cdiv(x_bits, 8),
                                 cudaMemcpyDeviceToDevice, xs));
        Prof pr(c, "decode_blocks", 1, s_gr.data_len + 8.0 * U, xs);
        launch_block_decode(at<uint32_t>(c, o_xpay), x_bits, U, at<uint8_t>(c, o_xw), at<uint8_t>(c, o_xk),
                            at<unsigned long long>(c, o_xoff), at<unsigned long long>(c, o_rv), SMALL_FIELD(c, err),
                            xs);
    }
    // A fixed-length -rle count stream sums the point count as it decodes (totals[0], zeroed on
    // its own stream first).
    bool counts_summed = false;
    for (auto& j : jobs)
        if (rle && j.slot == 3 && j.width == 4 && j.fixed_len && !j.fill) counts_summed = true;
    for (auto& j : jobs) {
        if (j.fill) {
            if (j.width == 1)
                launch_fill_u8(static_cast<uint8_t*>(j.out), j.nsym, static_cast<uint8_t>(j.fill_value), st);
            else
                launch_fill_u32(static_cast<uint32_t*>(j.out), j.nsym, static_cast<uint32_t>(j.fill_value), st);
            continue;
        }
        cudaStream_t js = side(c, j.slot);
        Prof pr(c, j.kind == kCodeGolombRice ? "decode_golomb_rice" : (j.kind == kCodeHuffman ? "decode_huffman" : "decode_exp_golomb"),
                1, j.total_bits / 8.0 + static_cast<double>(j.nsym) * j.width, js);
        if (j.fixed_len) {
            if (j.nsym * static_cast<uint64_t>(j.fixed_len) > j.total_bits)
                return fail(XNYZ_ERR_BAD_STREAM, "Huffman stream shorter than its symbols");
            const bool sum = counts_summed && j.slot == 3;
            if (sum) CUDA_TRY(cudaMemsetAsync(SMALL_FIELD(c, totals), 0, sizeof(unsigned long long) * 8, js));
            launch_decode_fixed(j.words, j.base_bits, j.total_bits, j.table, j.fixed_len, j.nsym, j.width, j.out,
                                SMALL_FIELD(c, err), js, sum ? SMALL_FIELD(c, totals[0]) : nullptr);
            continue;
        }
        // Golomb-Rice tracks k + 2 entry offsets per subsequence (derived in the kernel).
        const uint32_t* Lrun = nullptr;
        CUDA_TRY(cudaMemsetAsync(at<uint32_t>(c, o_dflag[j.slot]), 0, 4 * dtiles, js));
        launch_decode_stream(j.kind, j.words, j.base_bits, j.total_bits, j.table, j.L, Lrun, j.nsym, j.width, j.out,
                             at<uint32_t>(c, o_dflag[j.slot]), at<unsigned long long>(c, o_dagg[j.slot]),
                             at<unsigned long long>(c, o_dinc[j.slot]), SMALL_FIELD(c, tile_counters[30 + j.slot]),
                             SMALL_FIELD(c, err), SMALL_FIELD(c, fallback[j.slot]), SMALL_FIELD(c, codewords[j.slot]),
                             js);
    }
    CUDA_TRY(cudaGetLastError());
    TRY(join_sides(c));
    hd2.end();
    HostPhase hd3(c, "d3_decode_sync");
    // count total (for -rle) once the count stream is decoded; the fallback flags, totals,
    // codeword counts and the error word come back in one copy.  A stream whose parallel
    // decode gave up (rare) is decoded again sequentially and the counts re-summed.
    auto count_total = [&]() -> xnyz_status {
        if (!counts_summed) TRY(memset_small(c, offsetof(Small, totals), sizeof(unsigned long long) * 8, 0));
        if (rle && U && !counts_summed) {
            Prof pr(c, "count_total", 1, 4.0 * U);
            launch_count_total(at<int32_t>(c, o_counts), U, SMALL_FIELD(c, totals[0]), st);
        }
        CUDA_TRY(cudaGetLastError());
        return fetch_small(c, offsetof(Small, err), offsetof(Small, tile_counters) - offsetof(Small, err));
    };
    TRY(count_total());
    bool refetch = false;
    for (auto& j : jobs) {
        if (j.fill || j.fixed_len) continue;
        if (c->h_small->fallback[j.slot]) {
            launch_decode_sequential(j.kind, j.words, j.base_bits, j.total_bits, j.table, j.nsym, j.width, j.out,
                                     SMALL_FIELD(c, codewords[j.slot]), SMALL_FIELD(c, err), st);
            refetch = true;
        }
    }
    if (refetch) TRY(count_total());
    TRY(device_errors(c));
    for (auto& j : jobs)
        if (!j.fill && !j.fixed_len && c->h_small->codewords[j.slot] < j.nsym)
            return fail(XNYZ_ERR_BAD_STREAM, "stream " + std::to_string(j.slot) + " holds " +
                                                 std::to_string(c->h_small->codewords[j.slot]) + " codes, expected " +
                                                 std::to_string(j.nsym));
    if (!h.direct && NB && c->h_small->count_total != U)
        return fail(XNYZ_ERR_BAD_STREAM, "block counts do not add up to the point count");
    if (!h.direct && NB == 0 && U) return fail(XNYZ_ERR_BAD_STREAM, "no blocks");
    const uint64_t nout = (rle && !cells_out) ? c->h_small->totals[0] : U;
    hd3.end();
    HostPhase hd4(c, "d4_recover");

    // ---- output buffer (after the arena's planned part) ----
    Plan po;
    po.total = pl.total;
    const size_t o_out = po.add(12 * nout + 16);
    if (po.total > c->arena.cap) return fail(XNYZ_ERR_OOM, "__grow__:" + std::to_string(po.total));

    RecoverParams rp{};
    rp.q = q;
    rp.off[0] = h.off[0];
    rp.off[1] = h.off[1];
    rp.off[2] = h.off[2];
    // nx uses the size_t conversion of the stored int range (block_quantizer.hpp:163)
    rp.nx = static_cast<uint64_t>(static_cast<int64_t>(h.rx)) / 128 + 1;
    rp.ny = static_cast<uint64_t>(static_cast<int64_t>(h.ry)) / 128 + 1;
    rp.div_nx = make_u64div(rp.nx);
    rp.div_ny = make_u64div(rp.ny);
    rp.hilbert = h.hilbert;
    rp.hstart_inv = hm.inv_block_start;
    rp.rle = rle && !cells_out;
    rp.cells = cells_out != nullptr;
    rp.direct = h.direct;
    {
        int mr = std::max({h.rx, h.ry, h.rz}), bits = 0;
        for (int t = mr; t > 0; t >>= 1) ++bits;
        if (bits == 0) bits = 1;
        if (h.direct && bits > 20) return fail(XNYZ_ERR_UNSUPPORTED, "direct mode with more than 20 bits per axis");
        rp.bits = bits;
    }
    RecoverInputs ri{};
    ri.rep_sym = at<uint8_t>(c, o_rep);
    ri.rep_patch = at<unsigned long long>(c, o_patch);
    ri.npatch = P;
    ri.quad_sym = at<uint8_t>(c, o_quad);
    ri.is_start = at<uint8_t>(c, o_isst);
    ri.start_block = at<uint32_t>(c, o_stb);
    ri.blk_ids = at<unsigned long long>(c, o_blk);
    ri.nblocks = NB;
    ri.counts = at<int32_t>(c, o_counts);
    ri.rep_val = h.ext ? at<unsigned long long>(c, o_rv) : nullptr;
    CUDA_TRY(cudaMemsetAsync(at<uint32_t>(c, o_rflag), 0, 4 * rtiles * 5, st));
    float* out = at<float>(c, o_out);
    Prof pr_rec(c, "recover_units", 1,
                (h.direct ? 1.0 : 7.0) * U + 8.0 * P + (rle ? 4.0 * U : 0.0) + 12.0 * static_cast<double>(nout));
    launch_recover_units(ri, U, nout, rp, c->d_small->hil_inv, at<uint32_t>(c, o_rflag),
                         at<unsigned long long>(c, o_ragg), at<unsigned long long>(c, o_rinc),
                         SMALL_FIELD(c, tile_counters[40]), out, SMALL_FIELD(c, err), st);
    CUDA_TRY(cudaGetLastError());
    pr_rec.end();
    TRY(check_device_errors(c));
    *d_out = out;
    *n_out = nout;
    if (cells_out) *cells_out = at<int32_t>(c, o_counts);
    return XNYZ_OK;
}

xnyz_status decompress_run(xnyz_ctx* c, const uint8_t* d_cont, uint64_t len, const Header& h, int quantizer, float l2,
                           bool rle, size_t reserved, float** d_out, uint64_t* n_out, int32_t** cells_out = nullptr) {
    // The container may live in the arena's reserved prefix; growing keeps that prefix.
    for (int attempt = 0; attempt < 3; ++attempt) {
        xnyz_status s = decompress_core(c, d_cont, len, h, quantizer, l2, rle, reserved, d_out, n_out, cells_out);
        if (!(s == XNYZ_ERR_OOM && g_last_error.rfind("__grow__:", 0) == 0)) return s;
        const size_t need = std::stoull(g_last_error.substr(9));
        if (reserved) {
            char* old = c->arena.base;
            char* fresh = nullptr;
            const size_t cap = align_up(need + need / 8, 1 << 20);
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            CUDA_TRY(cudaMalloc(&fresh, cap));
            CUDA_TRY(cudaMemcpyAsync(fresh, old, reserved, cudaMemcpyDeviceToDevice, c->stream));
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            cudaFree(old);
            d_cont = reinterpret_cast<const uint8_t*>(fresh + (reinterpret_cast<const char*>(d_cont) - old));
            c->arena.base = fresh;
            c->arena.cap = cap;
        } else {
            TRY(ensure_arena(c, need));
        }
    }
    return fail(XNYZ_ERR_OOM, "workspace growth did not converge");
}

}  // namespace

namespace xnyz {
// An entry point reports only its own CUDA errors: a sticky error left on this thread by an
// earlier call outside the library (or by a call whose failure was already reported) is
// cleared first.
void clear_stale_cuda_error() { (void)cudaGetLastError(); }

// Sets the calling thread's xnyz_last_error() message (used by the batch pool).
xnyz_status set_last_error(xnyz_status s, const std::string& msg) { return fail(s, msg); }
}  // namespace xnyz

// ====================================================================== C ABI ==========
extern "C" {

const char* xnyz_last_error(void) { return g_last_error.c_str(); }
const char* xnyz_version(void) { return "xnyzip-b200 0.1 (sm_100a)"; }

xnyz_status xnyz_create(xnyz_ctx** out, int device, void* stream) {
    clear_stale_cuda_error();
    if (!out) return fail(XNYZ_ERR_INVALID_ARG, "null context pointer");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(XNYZ_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(XNYZ_ERR_INVALID_ARG, "device index out of range");
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(XNYZ_ERR_NO_DEVICE, "this build targets sm_100a (B200)");
    std::unique_ptr<xnyz_ctx> c(new xnyz_ctx());
    c->device = device;
    if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    CUDA_TRY(cudaMalloc(&c->d_small, sizeof(Small)));
    CUDA_TRY(cudaMemset(c->d_small, 0, sizeof(Small)));
    CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&c->h_small), sizeof(Small), cudaHostAllocDefault));
    std::memset(c->h_small, 0, sizeof(Small));
    CUDA_TRY(cudaEventCreate(&c->ev0));
    CUDA_TRY(cudaEventCreate(&c->ev1));
    CUDA_TRY(cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming));
    for (int k = 0; k < xnyz_ctx::kSide; ++k) {
        CUDA_TRY(cudaStreamCreateWithFlags(&c->side[k], cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&c->join_ev[k], cudaEventDisableTiming));
    }
    (void)hilbert_machines();
    *out = c.release();
    return XNYZ_OK;
}

xnyz_status xnyz_destroy(xnyz_ctx* c) {
    if (!c) return XNYZ_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->arena.base) cudaFree(c->arena.base);
    if (c->sort_status) cudaFree(c->sort_status);
    if (c->d_small) cudaFree(c->d_small);
    if (c->h_small) cudaFreeHost(c->h_small);
    if (c->h_stage) cudaFreeHost(c->h_stage);
    if (c->d_container) cudaFree(c->d_container);
    if (c->d_model) cudaFree(c->d_model);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (int k = 0; k < xnyz_ctx::kSide; ++k) {
        if (c->side[k]) {
            cudaStreamSynchronize(c->side[k]);
            cudaStreamDestroy(c->side[k]);
        }
        if (c->join_ev[k]) cudaEventDestroy(c->join_ev[k]);
    }
    if (c->fork_ev) cudaEventDestroy(c->fork_ev);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    (void)cudaGetLastError();  // teardown is best effort: leave no sticky error behind
    return XNYZ_OK;
}

xnyz_status xnyz_trim(xnyz_ctx* c) {
    clear_stale_cuda_error();
    if (!c) return fail(XNYZ_ERR_INVALID_ARG, "null context");
    cudaSetDevice(c->device);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->arena.base) cudaFree(c->arena.base);
    c->arena = Arena{};
    if (c->d_container) cudaFree(c->d_container);
    c->d_container = nullptr;
    c->d_container_cap = 0;
    return XNYZ_OK;
}

xnyz_status xnyz_set_zstd_library(const char* path) {
    std::string err;
    if (!zstd_load(path, err)) return fail(XNYZ_ERR_ZSTD, err);
    return XNYZ_OK;
}

xnyz_status xnyz_host_alloc(void** ptr, size_t bytes) {
    if (!ptr) return fail(XNYZ_ERR_INVALID_ARG, "null pointer");
    CUDA_TRY(cudaHostAlloc(ptr, bytes ? bytes : 1, cudaHostAllocDefault));
    return XNYZ_OK;
}
xnyz_status xnyz_host_free(void* ptr) {
    if (ptr) CUDA_TRY(cudaFreeHost(ptr));
    return XNYZ_OK;
}

void xnyz_free(void* p) { std::free(p); }

xnyz_status xnyz_compress(xnyz_ctx* c, const float* xyz, uint64_t n, int xyz_is_device, const xnyz_params* params,
                          int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order,
                          xnyz_compress_info* info) {
    clear_stale_cuda_error();
    if (!c || !xyz || !params || !out || !out_len) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    if (use_zstd) {
        std::string e;
        if (!zstd_available(e)) return fail(XNYZ_ERR_ZSTD, e);
    }
    cudaStream_t st = c->stream;
    CUDA_TRY(cudaEventRecord(c->ev0, st));
    const float* d_xyz = xyz;
    size_t reserved = 0;
    if (!xyz_is_device) {
        reserved = align_up(12 * n);
        const bool wo = sort_order != nullptr && !params->rle;
        TRY(ensure_arena(c, make_cplan(n, wo, reserved, c->block_mode != XNYZ_BLOCKS_OFF).total + encoder_reserve(n)));
        CUDA_TRY(cudaMemcpyAsync(c->arena.base, xyz, 12 * n, cudaMemcpyHostToDevice, st));
        d_xyz = reinterpret_cast<const float*>(c->arena.base);
    }
    CompressOut R;
    const bool want_order = sort_order != nullptr && !params->rle;
    TRY(compress_run(c, d_xyz, n, *params, want_order, reserved, R));
    // container: skeleton on the host, stream bytes copied from the device into place
    const size_t clen = R.cont.size;
    TRY(ensure_host_stage(c, clen));
    CUDA_TRY(R.cont.to_host(c->h_stage, st));
    std::vector<uint32_t> order;
    if (want_order) {
        order.resize(n);
        CUDA_TRY(cudaMemcpyAsync(order.data(), R.d_order, 4 * n, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaEventRecord(c->ev1, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (want_order)
        for (uint64_t i = 0; i < n; ++i) sort_order[i] = order[i];
    uint8_t* buf = nullptr;
    uint64_t blen = 0;
    HostPhase hz(c, "c8_zstd");
    if (use_zstd) {
        std::string e;
        const size_t cap = zstd_bound(clen);
        buf = static_cast<uint8_t*>(std::malloc(cap ? cap : 1));
        if (!buf) return fail(XNYZ_ERR_OOM, "host allocation");
        size_t w = 0;
        if (!zstd_compress_into(c->h_stage, clen, 3, buf, cap, w, e)) {
            std::free(buf);
            return fail(XNYZ_ERR_ZSTD, e);
        }
        blen = w;
    } else {
        buf = static_cast<uint8_t*>(std::malloc(clen ? clen : 1));
        if (!buf) return fail(XNYZ_ERR_OOM, "host allocation");
        std::memcpy(buf, c->h_stage, clen);
        blen = clen;
    }
    *out = buf;
    *out_len = blen;
    if (info) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        R.info.gpu_ms = ms;
        R.info.output_bytes = blen;
        *info = R.info;
    }
    return XNYZ_OK;
}

namespace {
// Sets the context's shared-codebook mode for one call and clears it afterwards.
struct ShareScope {
    xnyz_ctx* c;
    ShareScope(xnyz_ctx* cc, int mode) : c(cc) { c->share_mode = mode; }
    ~ShareScope() {
        c->share_mode = 0;
        c->share_rep.clear();
        c->share_quad.clear();
    }
};

// deserialize_profile (composer/block_encoding_profile.hpp:51-72), strict about sizes.
bool parse_profile(const uint8_t* p, uint64_t len, std::vector<uint8_t>& rep, std::vector<uint8_t>& quad) {
    uint64_t pos = 0;
    for (auto* dst : {&rep, &quad}) {
        if (pos + 4 > len) return false;
        const uint32_t n = uint32_t(p[pos]) | (uint32_t(p[pos + 1]) << 8) | (uint32_t(p[pos + 2]) << 16) |
                           (uint32_t(p[pos + 3]) << 24);
        pos += 4;
        if (n > len - pos) return false;
        dst->assign(p + pos, p + pos + n);
        pos += n;
    }
    return true;
}
}  // namespace

xnyz_status xnyz_fit_profile(xnyz_ctx* c, const float* xyz, uint64_t n, int xyz_is_device, const xnyz_params* params,
                             int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order, uint8_t** profile,
                             uint64_t* profile_len) {
    clear_stale_cuda_error();
    if (!c || !params || !profile || !profile_len) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    *profile = nullptr;
    *profile_len = 0;
    ShareScope scope(c, 1);
    TRY(xnyz_compress(c, xyz, n, xyz_is_device, params, use_zstd, out, out_len, sort_order, nullptr));
    uint8_t* p = static_cast<uint8_t*>(std::malloc(c->share_out.size()));
    if (!p) return fail(XNYZ_ERR_OOM, "host allocation");
    std::memcpy(p, c->share_out.data(), c->share_out.size());
    *profile = p;
    *profile_len = c->share_out.size();
    return XNYZ_OK;
}

xnyz_status xnyz_compress_with_profile(xnyz_ctx* c, const float* xyz, uint64_t n, int xyz_is_device,
                                       const xnyz_params* params, const uint8_t* profile, uint64_t profile_len,
                                       int use_zstd, uint8_t** out, uint64_t* out_len, uint64_t* sort_order) {
    clear_stale_cuda_error();
    if (!c || !params || (!profile && profile_len)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    ShareScope scope(c, 2);
    if (!profile || !parse_profile(profile, profile_len, c->share_rep, c->share_quad) || c->share_rep.empty() ||
        c->share_quad.empty())
        return fail(XNYZ_ERR_INVALID_ARG, "compress_with_profile: empty or malformed profile");
    return xnyz_compress(c, xyz, n, xyz_is_device, params, use_zstd, out, out_len, sort_order, nullptr);
}

xnyz_status xnyz_compress_device(xnyz_ctx* c, const float* xyz, uint64_t n, const xnyz_params* params,
                                 const uint8_t** dev_container, uint64_t* container_len, xnyz_compress_info* info) {
    clear_stale_cuda_error();
    if (!c || !xyz || !params || !dev_container || !container_len) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    CUDA_TRY(cudaEventRecord(c->ev0, st));
    CompressOut R;
    TRY(ensure_arena(c, make_cplan(n, false, 0, c->block_mode != XNYZ_BLOCKS_OFF).total + encoder_reserve(n)));
    TRY(compress_run(c, xyz, n, *params, false, 0, R));
    HostPhase hpa(c, "c7_assemble_device");
    const size_t clen = R.cont.size;
    if (c->d_container_cap < clen + 64) {
        CUDA_TRY(cudaStreamSynchronize(st));
        if (c->d_container) cudaFree(c->d_container);
        c->d_container = nullptr;
        const size_t want = align_up(clen + clen / 4 + 64, 1 << 20);
        CUDA_TRY(cudaMalloc(&c->d_container, want));
        c->d_container_cap = want;
    }
    TRY(ensure_host_stage(c, R.cont.blob.size()));
    CUDA_TRY(R.cont.to_device(c->d_container, c->h_stage, st));
    CUDA_TRY(cudaMemsetAsync(c->d_container + clen, 0, 64, st));
    CUDA_TRY(cudaEventRecord(c->ev1, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *dev_container = c->d_container;
    *container_len = clen;
    if (info) {
        float ms = 0;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        R.info.gpu_ms = ms;
        R.info.output_bytes = clen;
        *info = R.info;
    }
    return XNYZ_OK;
}

namespace {
// Host-buffer decompress: zstd + header on the host, decode on the device; the points stay
// in the context's arena (*d_out, *nout) for the caller to copy out.
xnyz_status decompress_host_input(xnyz_ctx* c, const uint8_t* in, uint64_t in_len, int is_zstd, int quantizer,
                                  float l2_bound, int rle, float** d_out, uint64_t* nout) {
    if (!c || !in) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (quantizer != XNYZ_QUANT_CUBE && quantizer != XNYZ_QUANT_TO && quantizer != XNYZ_QUANT_ADAPTIVE)
        return fail(XNYZ_ERR_INVALID_ARG, "quantizer must be 0 (cube), 1 (truncated octahedron) or 2 (adaptive)");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const uint8_t* raw = in;
    uint64_t len = in_len;
    std::string e;
    HostPhase hu(c, "d0_unzstd_header");
    if (is_zstd) {
        uint64_t fs = 0;
        if (!zstd_content_size(in, in_len, fs, e)) return fail(XNYZ_ERR_ZSTD, e);
        TRY(ensure_host_stage(c, fs + 64));
        if (!zstd_decompress(in, in_len, c->h_stage, fs, e)) return fail(XNYZ_ERR_ZSTD, e);
        raw = c->h_stage;
        len = fs;
    }
    Header h;
    TRY(parse_header([&](uint64_t off, uint64_t bytes, void* dst) { std::memcpy(dst, raw + off, bytes); return true; },
                     len, rle != 0, h));
    hu.end();
    const size_t reserved = align_up(len + 64);
    TRY(ensure_arena(c, reserved));
    CUDA_TRY(cudaMemcpyAsync(c->arena.base, raw, len, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(c->arena.base + len, 0, 64, st));
    return decompress_run(c, reinterpret_cast<const uint8_t*>(c->arena.base), len, h, quantizer, l2_bound, rle != 0,
                          reserved, d_out, nout);
}
}  // namespace

xnyz_status xnyz_decompress(xnyz_ctx* c, const uint8_t* in, uint64_t in_len, int is_zstd, int quantizer,
                            float l2_bound, int rle, float** xyz, uint64_t* n) {
    clear_stale_cuda_error();
    if (!xyz || !n) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    float* d_out = nullptr;
    uint64_t nout = 0;
    TRY(decompress_host_input(c, in, in_len, is_zstd, quantizer, l2_bound, rle, &d_out, &nout));
    cudaStream_t st = c->stream;
    HostPhase hdh(c, "d5_d2h");
    float* host = static_cast<float*>(std::malloc(12 * nout + 4));
    if (!host) return fail(XNYZ_ERR_OOM, "host allocation");
    // Through the pinned staging buffer in chunks (a pageable destination is slow to DMA to).
    const size_t total = 12 * nout, chunk = 64u << 20;
    TRY(ensure_host_stage(c, std::min(total, 2 * chunk) + 64));
    for (size_t off = 0, k = 0; off < total; off += chunk, ++k) {
        const size_t len = std::min(chunk, total - off);
        uint8_t* buf = c->h_stage + (k & 1) * chunk;
        CUDA_TRY(cudaMemcpyAsync(buf, reinterpret_cast<const uint8_t*>(d_out) + off, len, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        std::memcpy(reinterpret_cast<uint8_t*>(host) + off, buf, len);
    }
    *xyz = host;
    *n = nout;
    return XNYZ_OK;
}

xnyz_status xnyz_decompress_into(xnyz_ctx* c, const uint8_t* in, uint64_t in_len, int is_zstd, int quantizer,
                                 float l2_bound, int rle, float* xyz, uint64_t capacity, uint64_t* n) {
    clear_stale_cuda_error();
    if (!xyz || !n) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    float* d_out = nullptr;
    uint64_t nout = 0;
    TRY(decompress_host_input(c, in, in_len, is_zstd, quantizer, l2_bound, rle, &d_out, &nout));
    *n = nout;
    if (nout > capacity) return fail(XNYZ_ERR_INVALID_ARG, "output buffer too small (*n holds the point count)");
    HostPhase hdh(c, "d5_d2h");
    if (nout) CUDA_TRY(cudaMemcpyAsync(xyz, d_out, 12 * nout, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return XNYZ_OK;
}

xnyz_status xnyz_zstd_decompress_device(xnyz_ctx* c, uint64_t count, const uint8_t* const* dev_frames,
                                        const uint64_t* frame_len, uint8_t* const* dev_out, const uint64_t* out_cap,
                                        int64_t* out_len) {
    clear_stale_cuda_error();
    if (!c || (count && (!dev_frames || !frame_len || !dev_out || !out_cap || !out_len)))
        return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (count > (uint64_t)1 << 32)  // the workspace alone would be 600 TB; keeps the sizes below from wrapping
        return fail(XNYZ_ERR_INVALID_ARG, "too many frames in one call");
    CUDA_TRY(cudaSetDevice(c->device));
    if (!count) return XNYZ_OK;
    cudaStream_t st = c->stream;
    Plan pl;
    const size_t o_arr = pl.add(40 * count);  // src | src_len | dst | cap | out_len
    const size_t o_ws = pl.add(zstd_workspace_bytes() * count);
    TRY(ensure_arena(c, pl.total));
    TRY(ensure_host_stage(c, 40 * count));
    uint64_t* h = reinterpret_cast<uint64_t*>(c->h_stage);
    std::memcpy(h, dev_frames, 8 * count);
    std::memcpy(h + count, frame_len, 8 * count);
    std::memcpy(h + 2 * count, dev_out, 8 * count);
    std::memcpy(h + 3 * count, out_cap, 8 * count);
    uint64_t* d = at<uint64_t>(c, o_arr);
    CUDA_TRY(cudaMemcpyAsync(d, h, 32 * count, cudaMemcpyHostToDevice, st));
    launch_zstd_frames(reinterpret_cast<const uint8_t* const*>(d), d + count, reinterpret_cast<uint8_t* const*>(d + 2 * count),
                       d + 3 * count, reinterpret_cast<long long*>(d + 4 * count), at<char>(c, o_ws), count, st);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(h + 4 * count, d + 4 * count, 8 * count, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    uint64_t bad = count;
    for (uint64_t i = 0; i < count; ++i) {
        out_len[i] = static_cast<int64_t>(h[4 * count + i]);
        if (out_len[i] < 0 && bad == count) bad = i;
    }
    if (bad != count)
        return fail(XNYZ_ERR_BAD_STREAM, "zstd frame " + std::to_string(bad) + " did not decode (" +
                                             std::to_string(out_len[bad]) + ")");
    return XNYZ_OK;
}

xnyz_status xnyz_decompress_device(xnyz_ctx* c, const uint8_t* dev_container, uint64_t len, int quantizer,
                                   float l2_bound, int rle, const float** dev_xyz, uint64_t* n) {
    clear_stale_cuda_error();
    if (!c || !dev_container || !dev_xyz || !n) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (quantizer != XNYZ_QUANT_CUBE && quantizer != XNYZ_QUANT_TO && quantizer != XNYZ_QUANT_ADAPTIVE)
        return fail(XNYZ_ERR_INVALID_ARG, "quantizer must be 0 (cube), 1 (truncated octahedron) or 2 (adaptive)");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    // The kernels read up to 16 bytes past a stream's end; containers from
    // xnyz_compress_device carry 64 bytes of padding.  Others are copied into the arena.
    const uint8_t* d_cont = dev_container;
    size_t reserved = 0;
    if (dev_container != c->d_container) {
        reserved = align_up(len + 64);
        TRY(ensure_arena(c, reserved));
        CUDA_TRY(cudaMemcpyAsync(c->arena.base, dev_container, len, cudaMemcpyDeviceToDevice, st));
        CUDA_TRY(cudaMemsetAsync(c->arena.base + len, 0, 64, st));
        d_cont = reinterpret_cast<const uint8_t*>(c->arena.base);
    }
    Header h;
    HostPhase hph(c, "d0_header_device");
    // The header's fields are read through a 64 KB window of the container copied to the host
    // at once: a small container's whole header costs one copy, a large one a copy per stream
    // (each stream's lengths and meta follow the previous stream's data), instead of a copy
    // and a synchronisation per field.
    std::vector<uint8_t> win;
    uint64_t win_off = 0;
    xnyz_status s = parse_header(
        [&](uint64_t off, uint64_t bytes, void* dst) {
            if (win.empty() || off < win_off || off + bytes > win_off + win.size()) {
                const uint64_t want = std::min<uint64_t>(len - off, std::max<uint64_t>(bytes, 64u << 10));
                win.resize(want);
                win_off = off;
                if (cudaMemcpyAsync(win.data(), d_cont + off, want, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    return false;
            }
            std::memcpy(dst, win.data() + (off - win_off), bytes);
            return true;
        },
        len, rle != 0, h);
    if (s != XNYZ_OK) return s;
    hph.end();
    float* d_out = nullptr;
    uint64_t nout = 0;
    TRY(decompress_run(c, d_cont, len, h, quantizer, l2_bound, rle != 0, reserved, &d_out, &nout));
    CUDA_TRY(cudaStreamSynchronize(st));
    *dev_xyz = d_out;
    *n = nout;
    return XNYZ_OK;
}

// ---- distributed-RLE cell tables ------------------------------------------------------------
xnyz_status xnyz_encode_cells(xnyz_ctx* c, const int32_t* cells, const int32_t* counts, uint64_t n,
                              int cells_is_device, const int32_t* ranges, const float* offset, int hilbert,
                              int use_zstd, uint8_t** out, uint64_t* out_len) {
    clear_stale_cuda_error();
    if (!c || !cells || !counts || !ranges || !offset || !out || !out_len)
        return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (n == 0) return fail(XNYZ_ERR_INVALID_ARG, "no cells");
    CUDA_TRY(cudaSetDevice(c->device));
    if (use_zstd) {
        std::string e;
        if (!zstd_available(e)) return fail(XNYZ_ERR_ZSTD, e);
    }
    cudaStream_t st = c->stream;
    // host tables are staged in a buffer of their own (the workspace may move while it grows)
    int32_t* tmp = nullptr;
    struct Free {
        int32_t*& p;
        ~Free() {
            if (p) cudaFree(p);
        }
    } guard{tmp};
    CellInput ci{};
    if (cells_is_device) {
        ci.cells = cells;
        ci.counts = counts;
    } else {
        CUDA_TRY(cudaMalloc(&tmp, 16 * n));
        CUDA_TRY(cudaMemcpyAsync(tmp, cells, 12 * n, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(tmp + 3 * n, counts, 4 * n, cudaMemcpyHostToDevice, st));
        ci.cells = tmp;
        ci.counts = tmp + 3 * n;
    }
    for (int a = 0; a < 3; ++a) {
        ci.range[a] = ranges[a];
        ci.offset[a] = offset[a];
    }
    const xnyz_params p{XNYZ_QUANT_TO, 1.0f, hilbert ? 1 : 0, 1, 0};
    const int mode = c->block_mode;
    c->block_mode = XNYZ_BLOCKS_OFF;  // the reference's container
    CompressOut R;
    xnyz_status s = ensure_arena(c, make_cplan(n, true, 0, false).total + encoder_reserve(n));
    if (s == XNYZ_OK) s = compress_run(c, nullptr, n, p, true, 0, R, &ci);
    c->block_mode = mode;
    if (s != XNYZ_OK) return s;
    const size_t clen = R.cont.size;
    TRY(ensure_host_stage(c, clen));
    CUDA_TRY(R.cont.to_host(c->h_stage, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    size_t cap = use_zstd ? zstd_bound(clen) : clen;
    uint8_t* buf = static_cast<uint8_t*>(std::malloc(cap ? cap : 1));
    if (!buf) return fail(XNYZ_ERR_OOM, "host allocation");
    if (use_zstd) {
        std::string e;
        size_t w = 0;
        if (!zstd_compress_into(c->h_stage, clen, 3, buf, cap, w, e)) {
            std::free(buf);
            return fail(XNYZ_ERR_ZSTD, e);
        }
        cap = w;
    } else {
        std::memcpy(buf, c->h_stage, clen);
    }
    *out = buf;
    *out_len = cap;
    return XNYZ_OK;
}

xnyz_status xnyz_decompress_to_cells(xnyz_ctx* c, const uint8_t* in, uint64_t in_len, int is_zstd, int32_t** cells,
                                     int32_t** counts, uint64_t* n, float* offset, int32_t* ranges, int* hilbert) {
    clear_stale_cuda_error();
    if (!c || !in || !cells || !counts || !n || !offset || !ranges || !hilbert)
        return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    const uint8_t* raw = in;
    uint64_t len = in_len;
    std::string e;
    if (is_zstd) {
        uint64_t fs = 0;
        if (!zstd_content_size(in, in_len, fs, e)) return fail(XNYZ_ERR_ZSTD, e);
        TRY(ensure_host_stage(c, fs + 64));
        if (!zstd_decompress(in, in_len, c->h_stage, fs, e)) return fail(XNYZ_ERR_ZSTD, e);
        raw = c->h_stage;
        len = fs;
    }
    Header h;
    TRY(parse_header([&](uint64_t off, uint64_t bytes, void* dst) { std::memcpy(dst, raw + off, bytes); return true; },
                     len, true, h));
    if (h.direct) return fail(XNYZ_ERR_BAD_STREAM, "decompress_to_cells: a direct-mode container (cell tables use block mode)");
    if (h.ext) return fail(XNYZ_ERR_UNSUPPORTED, "decompress_to_cells: an extended container");
    const size_t reserved = align_up(len + 64);
    TRY(ensure_arena(c, reserved));
    CUDA_TRY(cudaMemcpyAsync(c->arena.base, raw, len, cudaMemcpyHostToDevice, st));
    CUDA_TRY(cudaMemsetAsync(c->arena.base + len, 0, 64, st));
    float* d_cells = nullptr;
    int32_t* d_counts = nullptr;
    uint64_t nu = 0;
    TRY(decompress_run(c, reinterpret_cast<const uint8_t*>(c->arena.base), len, h, XNYZ_QUANT_TO, 1.0f, true, reserved,
                       &d_cells, &nu, &d_counts));
    int32_t* hc = static_cast<int32_t*>(std::malloc(12 * nu + 4));
    int32_t* hk = static_cast<int32_t*>(std::malloc(4 * nu + 4));
    if (!hc || !hk) {
        std::free(hc);
        std::free(hk);
        return fail(XNYZ_ERR_OOM, "host allocation");
    }
    if (nu) {
        CUDA_TRY(cudaMemcpyAsync(hc, d_cells, 12 * nu, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(hk, d_counts, 4 * nu, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    *cells = hc;
    *counts = hk;
    *n = nu;
    for (int a = 0; a < 3; ++a) offset[a] = h.off[a];
    ranges[0] = h.rx;
    ranges[1] = h.ry;
    ranges[2] = h.rz;
    *hilbert = h.hilbert ? 1 : 0;
    return XNYZ_OK;
}

xnyz_status xnyz_expand_cells(xnyz_ctx* c, const int32_t* cells, const int32_t* counts, uint64_t n, int quantizer,
                              float l2_bound, const float* offset, float** xyz, uint64_t* n_points) {
    clear_stale_cuda_error();
    if (!c || (n && (!cells || !counts)) || !offset || !xyz || !n_points)
        return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (quantizer != XNYZ_QUANT_CUBE && quantizer != XNYZ_QUANT_TO && quantizer != XNYZ_QUANT_ADAPTIVE)
        return fail(XNYZ_ERR_INVALID_ARG, "quantizer must be 0 (cube), 1 (truncated octahedron) or 2 (adaptive)");
    // expand_cells_to_points recovers with the truncated octahedron or else the cube
    // quantizer (block_decompressor_rle.hpp:350-356)
    if (quantizer == XNYZ_QUANT_ADAPTIVE) quantizer = XNYZ_QUANT_CUBE;
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t st = c->stream;
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) total += counts[i] > 0 ? static_cast<uint64_t>(counts[i]) : 0;
    Plan pl;
    const size_t o_cells = pl.add(12 * n + 16), o_counts = pl.add(4 * n + 16), o_off = pl.add(16),
                 o_out = pl.add(12 * total + 16);
    const LB lb = plan_lb(pl, cdiv(std::max<uint64_t>(n, 1), 4096), 1);
    TRY(ensure_arena(c, pl.total));
    if (n) {
        CUDA_TRY(cudaMemcpyAsync(at<int32_t>(c, o_cells), cells, 12 * n, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaMemcpyAsync(at<int32_t>(c, o_counts), counts, 4 * n, cudaMemcpyHostToDevice, st));
    }
    CUDA_TRY(cudaMemcpyAsync(at<float>(c, o_off), offset, 12, cudaMemcpyHostToDevice, st));
    TRY(lb_clear(c, lb, 1));
    TRY(memset_small(c, offsetof(Small, err), sizeof(uint32_t), 0));
    TRY(memset_small(c, offsetof(Small, tile_counters), sizeof(uint32_t) * 64, 0));
    TRY(memset_small(c, offsetof(Small, totals), sizeof(unsigned long long) * 8, 0));
    launch_expand_cells(at<int32_t>(c, o_cells), at<int32_t>(c, o_counts), n, make_quant(quantizer, l2_bound),
                        at<float>(c, o_off), lb_state(c, lb), SMALL_FIELD(c, tile_counters[0]), at<float>(c, o_out),
                        total, SMALL_FIELD(c, totals[0]), SMALL_FIELD(c, err), st);
    CUDA_TRY(cudaGetLastError());
    TRY(check_device_errors(c));
    float* host = static_cast<float*>(std::malloc(12 * total + 4));
    if (!host) return fail(XNYZ_ERR_OOM, "host allocation");
    if (total) CUDA_TRY(cudaMemcpyAsync(host, at<float>(c, o_out), 12 * total, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    *xyz = host;
    *n_points = total;
    return XNYZ_OK;
}

// ---- extended container and the block-parameter predictor ---------------------------------
xnyz_status xnyz_set_block_mode(xnyz_ctx* c, int mode) {
    if (!c) return fail(XNYZ_ERR_INVALID_ARG, "null context");
    if (mode < XNYZ_BLOCKS_OFF || mode > XNYZ_BLOCKS_GLOBAL) return fail(XNYZ_ERR_INVALID_ARG, "unknown block mode");
    c->block_mode = mode;
    return XNYZ_OK;
}

uint64_t xnyz_model_param_count(void) { return kParamCount; }

xnyz_status xnyz_set_model(xnyz_ctx* c, const float* params, uint64_t count, float fallback_confidence) {
    clear_stale_cuda_error();
    if (!c || !params) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (count != static_cast<uint64_t>(kParamCount))
        return fail(XNYZ_ERR_INVALID_ARG, "expected " + std::to_string(kParamCount) + " parameters");
    if (!(fallback_confidence >= 0.0f && fallback_confidence <= 1.0f))
        return fail(XNYZ_ERR_INVALID_ARG, "fallback confidence must be in [0, 1]");
    CUDA_TRY(cudaSetDevice(c->device));
    if (!c->d_model) CUDA_TRY(cudaMalloc(&c->d_model, sizeof(float) * kParamCount));
    CUDA_TRY(cudaMemcpyAsync(c->d_model, params, sizeof(float) * kParamCount, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->fallback_conf = fallback_confidence;
    return XNYZ_OK;
}

xnyz_status xnyz_last_block_info(xnyz_ctx* c, xnyz_block_info* info) {
    if (!c || !info) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    *info = c->last_blocks;
    return XNYZ_OK;
}

xnyz_status xnyz_stage_repos(xnyz_ctx* c, const float* dev_xyz, uint64_t n, const xnyz_params* params,
                             uint64_t* dev_out, uint64_t cap, uint64_t* count) {
    clear_stale_cuda_error();
    if (!c || !dev_xyz || !params || !count || (cap && !dev_out)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    const int mode = c->block_mode;
    c->block_mode = XNYZ_BLOCKS_GLOBAL;
    const uint8_t* dc = nullptr;
    uint64_t dl = 0;
    const xnyz_status s = xnyz_compress_device(c, dev_xyz, n, params, &dc, &dl, nullptr);
    c->block_mode = mode;
    if (s != XNYZ_OK) return s;
    *count = c->last_repval_n;
    const uint64_t m = std::min(cap, c->last_repval_n);
    if (m) CUDA_TRY(cudaMemcpyAsync(dev_out, c->last_repval, 8 * m, cudaMemcpyDeviceToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return XNYZ_OK;
}

xnyz_status xnyz_block_features(const uint64_t* v, uint64_t n, float* feats, void* stream) {
    clear_stale_cuda_error();
    if (n && (!v || !feats)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    launch_block_features(reinterpret_cast<const unsigned long long*>(v), n, feats, static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}
xnyz_status xnyz_block_search(const uint64_t* v, uint64_t n, uint8_t* w, uint8_t* k, uint32_t* cost, void* stream) {
    clear_stale_cuda_error();
    if (n && (!v || !w || !k)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    launch_block_search(reinterpret_cast<const unsigned long long*>(v), n, nullptr, w, k, cost,
                        static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}
xnyz_status xnyz_block_cost(const uint64_t* v, uint64_t n, const uint8_t* w, const uint8_t* k, uint32_t* cost,
                            void* stream) {
    clear_stale_cuda_error();
    if (n && (!v || !w || !k || !cost)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    launch_block_cost(reinterpret_cast<const unsigned long long*>(v), n, w, k, cost, static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}
xnyz_status xnyz_mlp_forward(const float* prm, const float* feats, uint64_t count, uint8_t* w, uint8_t* k, float* conf,
                             float* logits, void* stream) {
    clear_stale_cuda_error();
    if (count && (!prm || !feats || !w || !k)) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    launch_mlp_forward(prm, feats, count, w, k, conf, logits, static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}
uint64_t xnyz_mlp_gather_floats(uint64_t count) { return mlp_gather_floats(count); }
xnyz_status xnyz_mlp_train_batch(const float* prm, const float* feats, const uint8_t* w, const uint8_t* k,
                                 const uint32_t* idx, uint64_t first, uint64_t count, float scale, float* grad,
                                 float* loss, float* gather, void* stream) {
    clear_stale_cuda_error();
    if (count && (!prm || !feats || !w || !k || !grad || !loss || !gather))
        return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    launch_mlp_train(prm, feats, w, k, idx, first, count, scale, grad, loss, gather, static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}
xnyz_status xnyz_mlp_adam(float* prm, float* grad, float* m, float* v, float lr, int step, void* stream) {
    clear_stale_cuda_error();
    if (!prm || !grad || !m || !v || step < 1) return fail(XNYZ_ERR_INVALID_ARG, "bad argument");
    launch_mlp_adam(prm, grad, m, v, lr, step, static_cast<cudaStream_t>(stream));
    CUDA_TRY(cudaGetLastError());
    return XNYZ_OK;
}

// ---- stage entry points -------------------------------------------------------------------
xnyz_status xnyz_stage_quantize(xnyz_ctx* c, const float* dev_xyz, uint64_t n, int quantizer, float l2_bound,
                                float* offset3, int32_t* dev_cells) {
    clear_stale_cuda_error();
    if (!c || !dev_xyz || !offset3 || !dev_cells || n == 0) return fail(XNYZ_ERR_INVALID_ARG, "bad argument");
    if (quantizer != XNYZ_QUANT_CUBE && quantizer != XNYZ_QUANT_TO)
        return fail(XNYZ_ERR_INVALID_ARG, "stage quantizer must be 0 (cube) or 1 (truncated octahedron)");
    CUDA_TRY(cudaSetDevice(c->device));
    const QuantParams q = make_quant(quantizer, l2_bound);
    PointStats init{};
    for (int a = 0; a < 3; ++a) {
        init.minkey[a] = ~0ull;
        init.min_cell[a] = INT32_MAX;
    }
    c->h_small->stats = init;
    CUDA_TRY(cudaMemcpyAsync(&c->d_small->stats, &c->h_small->stats, sizeof(PointStats), cudaMemcpyHostToDevice, c->stream));
    launch_bbox(dev_xyz, n, SMALL_FIELD(c, stats), c->stream);
    launch_quantize_range(dev_xyz, n, q, SMALL_FIELD(c, stats), 0, c->stream);
    launch_quantize_cells(dev_xyz, n, q, SMALL_FIELD(c, stats), dev_cells, c->stream);
    CUDA_TRY(cudaGetLastError());
    TRY(fetch_small(c, offsetof(Small, stats), sizeof(PointStats)));
    for (int a = 0; a < 3; ++a) offset3[a] = c->h_small->stats.offset[a];
    return XNYZ_OK;
}

xnyz_status xnyz_stage_recover(xnyz_ctx* c, const int32_t* dev_cells, uint64_t n, int quantizer, float l2_bound,
                               const float* offset3, float* dev_xyz) {
    clear_stale_cuda_error();
    if (!c || !dev_cells || !offset3 || !dev_xyz) return fail(XNYZ_ERR_INVALID_ARG, "bad argument");
    if (quantizer != XNYZ_QUANT_CUBE && quantizer != XNYZ_QUANT_TO)
        return fail(XNYZ_ERR_INVALID_ARG, "stage quantizer must be 0 (cube) or 1 (truncated octahedron)");
    CUDA_TRY(cudaSetDevice(c->device));
    for (int a = 0; a < 3; ++a) c->h_small->offset_in[a] = offset3[a];
    CUDA_TRY(cudaMemcpyAsync(c->d_small->offset_in, c->h_small->offset_in, 12, cudaMemcpyHostToDevice, c->stream));
    launch_recover_cells(dev_cells, n, make_quant(quantizer, l2_bound), c->d_small->offset_in, dev_xyz, c->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return XNYZ_OK;
}

xnyz_status xnyz_stage_hilbert(xnyz_ctx* c, const uint64_t* dev_in, uint64_t n, unsigned iteration, int inverse,
                               uint64_t* dev_out) {
    clear_stale_cuda_error();
    if (!c || !dev_in || !dev_out) return fail(XNYZ_ERR_INVALID_ARG, "bad argument");
    if (iteration > 20) return fail(XNYZ_ERR_UNSUPPORTED, "iteration above 20");
    CUDA_TRY(cudaSetDevice(c->device));
    const auto& hm = hilbert_machines();
    uint8_t* tab = inverse ? c->d_small->hil_inv : c->d_small->hil_fwd;
    CUDA_TRY(cudaMemcpyAsync(tab, inverse ? hm.inv.data() : hm.fwd.data(), 256, cudaMemcpyHostToDevice, c->stream));
    launch_hilbert(reinterpret_cast<const unsigned long long*>(dev_in), n, tab, static_cast<int>(iteration), 0u,
                   reinterpret_cast<unsigned long long*>(dev_out), c->stream);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return XNYZ_OK;
}

xnyz_status xnyz_stage_sort(xnyz_ctx* c, uint64_t* dev_keys, uint32_t* dev_payload, uint64_t n, int key_bits) {
    clear_stale_cuda_error();
    if (!c || !dev_keys || key_bits < 0 || key_bits > 64) return fail(XNYZ_ERR_INVALID_ARG, "bad argument");
    if (n >= (1ull << 31)) return fail(XNYZ_ERR_UNSUPPORTED, "more than 2^31 - 1 keys");
    CUDA_TRY(cudaSetDevice(c->device));
    const int passes = static_cast<int>(cdiv(key_bits, 8));
    if (passes == 0 || n <= 1) return XNYZ_OK;
    Plan pl;
    const size_t ok = pl.add(8 * n), ov = pl.add(4 * n);
    TRY(ensure_arena(c, pl.total));
    SortBufs sb{{reinterpret_cast<unsigned long long*>(dev_keys), at<unsigned long long>(c, ok)},
                {dev_payload, dev_payload ? at<uint32_t>(c, ov) : nullptr}};
    TRY(memset_small(c, offsetof(Small, sort_hist), sizeof(uint32_t) * 8 * 256, 0));
    TRY(memset_small(c, offsetof(Small, err), sizeof(uint32_t), 0));
    launch_sort_histogram(sb.keys[0], n, passes, c->d_small->sort_hist, c->stream);
    int res = 0;
    TRY(radix_sort(c, sb, n, passes, c->d_small->sort_hist, res));
    if (res) {
        CUDA_TRY(cudaMemcpyAsync(dev_keys, sb.keys[1], 8 * n, cudaMemcpyDeviceToDevice, c->stream));
        if (dev_payload) CUDA_TRY(cudaMemcpyAsync(dev_payload, sb.vals[1], 4 * n, cudaMemcpyDeviceToDevice, c->stream));
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return check_device_errors(c);
}

xnyz_status xnyz_profile(xnyz_ctx* c, int enable) {
    if (!c) return fail(XNYZ_ERR_INVALID_ARG, "null context");
    c->prof = enable != 0;
    c->serial = enable == 2;
    c->prof_recs.clear();
    c->host_ms.clear();
    c->ev_used = 0;
    return XNYZ_OK;
}

xnyz_status xnyz_profile_read(xnyz_ctx* c, char* json, uint64_t cap, uint64_t* len) {
    clear_stale_cuda_error();
    if (!c || !len) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    struct Agg {
        double ms = 0, bytes = 0;
        uint64_t launches = 0, calls = 0;
    };
    std::map<std::string, Agg> agg;
    for (const auto& r : c->prof_recs) {
        float ms = 0;
        CUDA_TRY(cudaEventElapsedTime(&ms, r.a, r.b));
        Agg& a = agg[r.name];
        a.ms += ms;
        a.bytes += r.bytes;
        a.launches += r.launches;
        a.calls += 1;
    }
    std::string out = "{";
    bool first = true;
    for (const auto& kv : agg) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s\"%s\": {\"ms\": %.6f, \"launches\": %llu, \"calls\": %llu, \"bytes\": %.1f}",
                      first ? "" : ", ", kv.first.c_str(), kv.second.ms,
                      static_cast<unsigned long long>(kv.second.launches),
                      static_cast<unsigned long long>(kv.second.calls), kv.second.bytes);
        out += buf;
        first = false;
    }
    for (const auto& kv : c->host_ms) {
        char buf[256];
        std::snprintf(buf, sizeof(buf), "%s\"host:%s\": {\"ms\": %.6f, \"launches\": 0, \"calls\": %llu, \"bytes\": 0}",
                      first ? "" : ", ", kv.first.c_str(), kv.second.first,
                      static_cast<unsigned long long>(kv.second.second));
        out += buf;
        first = false;
    }
    out += "}";
    *len = out.size();
    if (json && cap) {
        const size_t k = std::min<size_t>(cap - 1, out.size());
        std::memcpy(json, out.data(), k);
        json[k] = 0;
    }
    c->prof_recs.clear();
    c->host_ms.clear();
    c->ev_used = 0;
    return XNYZ_OK;
}

xnyz_status xnyz_host_hilbert(const uint64_t* in, uint64_t n, unsigned iteration, int inverse, uint64_t* out) {
    if ((!in || !out) && n) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    if (iteration > 20) return fail(XNYZ_ERR_UNSUPPORTED, "iteration above 20");
    const auto& hm = hilbert_machines();
    for (uint64_t i = 0; i < n; ++i)
        out[i] = hilbert_apply_host(inverse ? hm.inv : hm.fwd, in[i], static_cast<int>(iteration), 0u);
    return XNYZ_OK;
}

xnyz_status xnyz_host_codebook(int symtype, int count_stream, const uint64_t* symbols, const uint64_t* counts,
                               const uint64_t* first_index, uint64_t nsyms, uint64_t total, uint8_t* meta,
                               uint64_t* meta_len, uint64_t* encoded_bits, int* exp_golomb) {
    if ((nsyms && (!symbols || !counts || !first_index)) || !meta_len) return fail(XNYZ_ERR_INVALID_ARG, "null argument");
    std::vector<SymbolStat> st(nsyms);
    for (uint64_t i = 0; i < nsyms; ++i) st[i] = SymbolStat{symbols[i], counts[i], first_index[i]};
    const SymType t = symtype == 0 ? SymType::U64 : (symtype == 1 ? SymType::U8 : SymType::I32);
    const StreamCode sc = count_stream ? build_count_code(st, total) : build_stream_code(t, st, total);
    const uint64_t cap = *meta_len;
    *meta_len = sc.meta.size();
    if (meta && cap) std::memcpy(meta, sc.meta.data(), std::min<uint64_t>(cap, sc.meta.size()));
    if (encoded_bits) *encoded_bits = sc.encoded_bits;
    if (exp_golomb) *exp_golomb = sc.exp_golomb;
    return XNYZ_OK;
}

}  // extern "C"
