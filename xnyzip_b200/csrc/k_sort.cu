// Stable LSD radix sort of 64-bit keys (optional 32-bit payload), one 8-bit digit per pass,
// single-pass ("onesweep") scatter with decoupled look-back over tiles of 4096 keys.
//
// Replaces radix_sort + the per-id std::sort of quantizer/block_quantizer.hpp:33-76 and the
// std::sort of (sfc, index) pairs of composer/block_compressor.hpp:103: the keys packed by
// the key kernels order exactly as (id, reid) resp. (sfc, index) do, and only the digits
// that can be non-zero are sorted.
//
// Per pass: each warp ranks its 512 keys against warp-private digit counters, finding the
// lanes that share a digit through a per-warp bit mask in shared memory (one atomicOr per
// lane: cheaper than match.any, which serialises on the address-divergence pipe), the
// block turns warp counts into tile-local digit offsets, one thread per digit publishes the
// tile's count and starts the look-back over the previous tiles' digit counts (two
// predecessors per step; epoch-tagged 64-bit status words, so the status array is never
// cleared between passes), the keys are staged in shared memory in digit order while those
// loads are in flight, and, once the look-back has resolved the tile's global bases, written
// out in coalesced runs.
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096
constexpr int kWarps = kThreads / 32;
constexpr int kRadix = 256;
static_assert(kTile == kSortTile, "tile size");

// status word: [63:50] epoch, [49:48] flag (1 aggregate, 2 inclusive), [47:0] count
__device__ __forceinline__ u64 pack_status(u32 epoch, u32 flag, u64 count) {
    return ((u64)epoch << 50) | ((u64)flag << 48) | (count & ((1ull << 48) - 1));
}

// Look-back of digit d over the previous tiles' status words, kLookWindow predecessors per
// step (their loads in flight together).  `pre` holds the first window, loaded by the caller
// before it stages the tile's keys, so that the wait overlaps that work.  Publishes the
// tile's inclusive count and returns the count of digit d in all previous tiles.
constexpr int kLookWindow = 2;

__device__ u64 digit_lookback(u64* status, u32 tile, u32 d, u64 count, u32 epoch, u32* err, const u64* pre0) {
    u64 acc = 0;
    long long t = (long long)tile - 1;
    u64 pre[kLookWindow];
#pragma unroll
    for (int q = 0; q < kLookWindow; ++q) pre[q] = pre0[q];
    u32 spins = 0;
    while (t >= 0) {
        int used = 0;
        bool done = false;
#pragma unroll
        for (int q = 0; q < kLookWindow; ++q) {
            if (done || t - q < 0) break;
            const u64 s = pre[q];
            const u32 e = (u32)(s >> 50), f = (u32)(s >> 48) & 3u;
            if (e != epoch || f == 0) break;  // not published yet: re-read from here
            acc += s & ((1ull << 48) - 1);
            ++used;
            if (f == 2) done = true;
        }
        if (done) break;
        if (used == 0) {
            if (++spins > kSpinLimit) {
                atomicOr(err, kErrTimeout);
                break;
            }
            if (spins > 8) __nanosleep(32);
        }
        t -= used;
#pragma unroll
        for (int q = 0; q < kLookWindow; ++q)
            pre[q] = t - q >= 0 ? ld_volatile(&status[(u64)(t - q) * kRadix + d]) : 0ull;
    }
    st_volatile(&status[(u64)tile * kRadix + d], pack_status(epoch, 2, acc + count));
    return acc;
}

// Keys only: 4 CTAs per SM (64 registers, 52 KB shared); with payload: 3.
template <bool PAYLOAD>
__global__ void __launch_bounds__(kThreads, PAYLOAD ? 3 : 4) sort_pass_kernel(const u64* __restrict__ kin, u64* __restrict__ kout,
                                                             const u32* __restrict__ vin, u32* __restrict__ vout,
                                                             u64 n, int shift, const u32* __restrict__ offsets,
                                                             u64* status, u32 epoch, u32* tile_counter, u32* err) {
    extern __shared__ __align__(16) unsigned char smem[];
    u64* skeys = reinterpret_cast<u64*>(smem);                                  // kTile
    u64* gbase = skeys + kTile;                                                 // kRadix
    u32* whist = reinterpret_cast<u32*>(gbase + kRadix);                        // kWarps * kRadix
    u32* dstart = whist + kWarps * kRadix;                                      // kRadix
    u32* scratch = dstart + kRadix;                                             // 16
    u32* slot = scratch + 16;                                                   // 1
    u32* dmask = slot + 16;                                                     // kWarps * kRadix
    u32* svals = dmask + kWarps * kRadix;                                       // kTile (PAYLOAD)

    const u32 tile = claim_tile(tile_counter, slot);
    const u64 base = (u64)tile * kTile;
    const int tid = threadIdx.x, w = tid >> 5, lane = lane_id();
    for (int i = tid; i < kWarps * kRadix; i += kThreads) {
        whist[i] = 0;
        dmask[i] = 0;
    }
    __syncthreads();

    u64 k[kItems];
    u32 v[kItems];
    u32 rank[kItems];
    const u64 wbase = base + (u64)w * (32 * kItems);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const u64 j = wbase + (u64)i * 32 + lane;
        const bool ok = j < n;
        k[i] = ok ? kin[j] : 0ull;
        if (PAYLOAD) v[i] = ok ? vin[j] : 0u;
    }
    u32* wh = whist + w * kRadix;
    u32* wm = dmask + w * kRadix;
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        const bool ok = wbase + (u64)i * 32 + lane < n;
        const u32 d = (u32)(k[i] >> shift) & 255u;
        if (ok) atomicOr(&wm[d], 1u << lane);
        __syncwarp();
        u32 peers = 0, prev = 0;
        if (ok) {
            peers = wm[d];
            prev = wh[d];
        }
        __syncwarp();
        if (ok && (u32)lane == (u32)(__ffs(peers) - 1)) {
            wh[d] = prev + __popc(peers);
            wm[d] = 0;
        }
        __syncwarp();
        rank[i] = prev + __popc(peers & lanemask_lt());
    }
    __syncthreads();

    // Digit d (thread d): exclusive offsets of the warps, tile count, tile-local start.
    u32 tile_count;
    {
        const int d = tid;
        u32 s = 0;
#pragma unroll
        for (int ww = 0; ww < kWarps; ++ww) {
            const u32 c = whist[ww * kRadix + d];
            whist[ww * kRadix + d] = s;
            s += c;
        }
        tile_count = s;
    }
    u32 total;
    const u32 start = block_exclusive<kThreads>(tile_count, 0u, AddOp{}, scratch, total);
    dstart[tid] = start;
    // Digit tid: publish the tile's count and load the first look-back window; the keys are
    // staged while those loads are in flight, then the look-back completes.
    u64 pre[kLookWindow];
    if (tile == 0) {
        st_volatile(&status[tid], pack_status(epoch, 2, tile_count));
    } else {
        st_volatile(&status[(u64)tile * kRadix + tid], pack_status(epoch, 1, tile_count));
#pragma unroll
        for (int q = 0; q < kLookWindow; ++q)
            pre[q] = (long long)tile - 1 - q >= 0 ? ld_volatile(&status[(u64)(tile - 1 - q) * kRadix + tid]) : 0ull;
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (wbase + (u64)i * 32 + lane < n) {
            const u32 d = (u32)(k[i] >> shift) & 255u;
            const u32 p = dstart[d] + whist[w * kRadix + d] + rank[i];
            skeys[p] = k[i];
            if (PAYLOAD) svals[p] = v[i];
        }
    }
    const u64 before = tile == 0 ? 0ull : digit_lookback(status, tile, (u32)tid, tile_count, epoch, err, pre);
    gbase[tid] = (u64)offsets[tid] + before - dstart[tid];  // + tile slot p: the output position (u64, wrapping)
    __syncthreads();

    const u32 cnt = (u32)min((u64)kTile, n - base);
    for (u32 p = tid; p < cnt; p += kThreads) {
        const u64 key = skeys[p];
        const u32 d = (u32)(key >> shift) & 255u;
        const u64 o = gbase[d] + p;
        if (o >= n) {  // only after an expired look-back wait: flagged, never written
            atomicOr(err, kErrPlacement);
            continue;
        }
        kout[o] = key;
        if (PAYLOAD) vout[o] = svals[p];
    }
}

constexpr size_t smem_bytes(bool payload) {
    return kTile * 8 + kRadix * 8 + kWarps * kRadix * 4 + kRadix * 4 + 32 * 4 + kWarps * kRadix * 4 +
           (payload ? kTile * 4 : 0);
}

__global__ void __launch_bounds__(kThreads) histogram_kernel(const u64* __restrict__ keys, u64 n, int passes,
                                                             u32* hist) {
    __shared__ u32 sh[8 * kRadix];
    for (int i = threadIdx.x; i < passes * kRadix; i += kThreads) sh[i] = 0;
    __syncthreads();
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 j = (u64)blockIdx.x * kThreads + threadIdx.x; j < n; j += stride) {
        const u64 key = keys[j];
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p * kRadix + (u32)((key >> (8 * p)) & 255u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * kRadix; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// One block per pass: digit counts -> exclusive digit offsets, in place.
__global__ void __launch_bounds__(kRadix) offsets_kernel(u32* hist) {
    __shared__ u32 scratch[16];
    u32* h = hist + blockIdx.x * kRadix;
    const u32 c = h[threadIdx.x];
    u32 total;
    const u32 e = block_exclusive<kRadix>(c, 0u, AddOp{}, scratch, total);
    h[threadIdx.x] = e;
}

}  // namespace

void launch_sort_histogram(const unsigned long long* keys, uint64_t n, int passes, uint32_t* hist, cudaStream_t st) {
    u64 blocks = (n + kThreads - 1) / kThreads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    histogram_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(keys, n, passes, hist);
}

void launch_sort_offsets(uint32_t* hist, int passes, cudaStream_t st) {
    offsets_kernel<<<passes, kRadix, 0, st>>>(hist);
}

void launch_sort_pass(const unsigned long long* kin, unsigned long long* kout, const uint32_t* vin, uint32_t* vout,
                      uint64_t n, int shift, const uint32_t* offsets, unsigned long long* status, uint32_t epoch,
                      uint32_t* tile_counter, uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (tiles == 0) return;
    // The dynamic shared-memory limit is a per-device function attribute; setting it on
    // every launch keeps multi-device use correct and costs a few microseconds.
    if (vin) {
        cudaFuncSetAttribute(sort_pass_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes(true));
        sort_pass_kernel<true><<<tiles, kThreads, smem_bytes(true), st>>>(kin, kout, vin, vout, n, shift, offsets,
                                                                          status, epoch, tile_counter, err);
    } else {
        cudaFuncSetAttribute(sort_pass_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_bytes(false));
        sort_pass_kernel<false><<<tiles, kThreads, smem_bytes(false), st>>>(kin, kout, nullptr, nullptr, n, shift,
                                                                           offsets, status, epoch, tile_counter, err);
    }
}

}  // namespace dev
}  // namespace xnyz
