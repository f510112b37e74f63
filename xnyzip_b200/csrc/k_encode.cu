// Compress-side stream kernels over the sorted keys.
//
//   units_*       one pass over the sorted keys: RLE run heads (unique cells), block heads,
//                 quad / repos deltas (block mode) or SFC deltas (direct mode), PFor symbols
//                 and patches, symbol histograms with first-occurrence units, all placed by
//                 a three-channel chained scan (units, patches, blocks).
//   count_stats   -rle count per unit and its histogram.
//   block_deltas  + bitpack: BitPacker<uint64_t> of the block-id and block-count deltas.
//   gr_encode     GolombRiceCoder<uint64_t>::pack of the patches.
//   huff_encode_* HuffmanEncoder<T>::encode / exp-Golomb encode with host-built codes.
//
// Reference (paths relative to its source/): quantizer/block_quantizer.hpp:117-149 (LCP
// streams), composer/block_compressor.hpp:110-114,146-147 (deltas), encoder/
// p_for_delta_encoder.hpp:27-43 (PFor, limit 254), encoder/golomb_rice_encoder.hpp:92-148,
// encoder/bitpacking_encoder.hpp:17-51, encoder/huffman_encoder.hpp:150-170,365-396,
// composer/block_compressor_rle.hpp:97-123,290-308 (dedup and count stream).
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
static_assert(kTile == kUnitTile && kTile == kEncTile, "tile size");

__device__ __forceinline__ void block_key_fields(u64 k, const BlockKeyParams& kp, u64& id, u32& quad, u32& sfc) {
    id = (kp.defect_flag && k >= kp.defect_flag) ? (((k - kp.defect_flag) >> 21) + kp.defect_base) : (k >> 21);
    quad = (u32)(k >> 18) & 7u;
    sfc = (u32)(k & 0x3ffffu);
}

__device__ __forceinline__ u64 direct_key_sfc(u64 k, const DirectKeyParams& kp) {
    return (kp.defect_flag && k >= kp.defect_flag) ? (kp.defect_high | (k - kp.defect_flag)) : k;
}

// Warp-aggregated histogram update with first-occurrence tracking; the lowest lane of a
// group of equal symbols holds the smallest unit index (units grow with the lane).
__device__ __forceinline__ void hist_add(u32* hist, u32* first, bool valid, u32 sym, u32 unit) {
    const u32 peers = __match_any_sync(kFullMask, valid ? sym : (0x10000u | lane_id()));
    if (valid && lane_id() == (u32)(__ffs(peers) - 1)) {
        atomicAdd(&hist[sym], (u32)__popc(peers));
        atomicMin(&first[sym], unit);
    }
}

// The same update with the groups of equal symbols found through a per-warp bit mask in
// shared memory (one atomicOr per lane) instead of match.any, which serialises on the
// address-divergence pipe.  `masks` is zero on entry and on return.
__device__ __forceinline__ void hist_add_masked(u32* masks, u32* hist, u32* first, bool valid, u32 sym, u32 unit) {
    const u32 lane = lane_id();
    if (valid) atomicOr(&masks[sym], 1u << lane);
    __syncwarp();
    if (valid) {
        const u32 peers = masks[sym];
        if (lane == (u32)(__ffs(peers) - 1)) {
            atomicAdd(&hist[sym], (u32)__popc(peers));
            atomicMin(&first[sym], unit);
        }
    }
    __syncwarp();
    if (valid) masks[sym] = 0u;
    __syncwarp();
}

template <bool DIRECT>
__global__ void __launch_bounds__(kThreads) units_kernel(const u64* __restrict__ keys, u64 n, int rle,
                                                         BlockKeyParams bkp, DirectKeyParams dkp, UnitOutputs out,
                                                         LookBackState lb, u32* tile_counter, u32* err) {
    __shared__ u64 sk[kTile + 1];
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase[3];
    __shared__ u32 hrep[256], frep[256], hquad[16], fquad[16];
    __shared__ u32 mrep[kThreads / 32][256];
    __shared__ u64 psum[kThreads / 32];

    const u32 tile = claim_tile(tile_counter, &slot);
    const u32 ntiles = gridDim.x;
    const u64 base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, n - base);
    const int tid = threadIdx.x;
    if (tid == 0) sk[0] = base ? keys[base - 1] : 0ull;
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + tid;
        if (e < cnt) sk[1 + e] = keys[base + e];
    }
    hrep[tid] = 0;
    frep[tid] = 0xffffffffu;
    if (tid < 16) {
        hquad[tid] = 0;
        fquad[tid] = 0xffffffffu;
    }
    for (int i = tid; i < (kThreads / 32) * 256; i += kThreads) (&mrep[0][0])[i] = 0u;
    __syncthreads();

    // Element e of the tile: flags (bit0 head, bit1 patch, bit2 new block, bits 8..15 quad
    // delta), repos / SFC delta and block id.  Computed in pass A for the counts and again in
    // pass B from the staged keys (cheaper than holding 16 of each in registers).
    auto classify = [&](u32 e, u64& val, u64& idv) -> u32 {
        val = 0;
        idv = 0;
        if (e >= cnt) return 0u;
        const u64 j = base + e;
        const u64 k = sk[1 + e], kp = sk[e];
        const bool head = !rle || j == 0 || k != kp;
        if (!head) return 0u;
        u32 f = 1u;
        if (DIRECT) {
            const u64 s = direct_key_sfc(k, dkp);
            const u64 d = j == 0 ? s : s - direct_key_sfc(kp, dkp);
            val = d;
            if (d > 254u) f |= 2u;
        } else {
            u64 id, idp = 0;
            u32 quad, sfc, quadp = 0, sfcp = 0;
            block_key_fields(k, bkp, id, quad, sfc);
            if (j > 0) block_key_fields(kp, bkp, idp, quadp, sfcp);
            const bool nb = (j == 0) || id != idp;
            u32 qd;
            u64 r;
            if (nb) {
                qd = quad;
                r = sfc;
                f |= 4u;
            } else if (quad != quadp) {
                qd = quad - quadp;
                r = sfc;
            } else {
                qd = 0;
                r = (u64)sfc - (u64)sfcp;
            }
            val = r;
            idv = id;
            if (r > 254u) f |= 2u;
            f |= (qd & 0xffu) << 8;
        }
        return f;
    };
    // Warp w owns elements [512 w, 512 w + 512) of the tile, taken 32 consecutive elements
    // (one per lane) per round: staged keys are read without bank conflicts, and the
    // outputs of a round land in consecutive units, so the stores coalesce.
    const int w = tid >> 5;
    const u32 lane = lane_id();
    const u32 wfirst = (u32)w * (32u * kItems);
    // Pass A: count heads, patches and new blocks of my 16 elements.
    u32 h = 0, p = 0, b = 0;
    for (int r = 0; r < kItems; ++r) {
        u64 v, id;
        const u32 f = classify(wfirst + (u32)r * 32u + lane, v, id);
        h += f & 1u;
        p += (f >> 1) & 1u;
        b += (f >> 2) & 1u;
    }
    // Packed three-field exclusive scan: each field <= 4096 per tile, 21 bits apiece.  Lane
    // 0's exclusive prefix is the count over the earlier warps' elements.
    const u64 mine = (u64)h | ((u64)p << 21) | ((u64)b << 42);
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(mine, 0ull, AddOp{}, scratch, tot);
    if (tid < 96) {  // warps 0, 1, 2: one chained scan each
        const int ch = tid >> 5;
        const u64 part = (tot >> (21 * ch)) & ((1ull << 21) - 1);
        LookBack64 l{lb.flag + ch * ntiles, lb.agg + ch * ntiles, lb.inc + ch * ntiles};
        const u64 before = warp_lookback_add(l, tile, part, err);
        if ((tid & 31) == 0) {
            sbase[ch] = before;
            if (tile == ntiles - 1) out.counters[ch] = before + part;
        }
    }
    __syncthreads();

    const u64 wex = __shfl_sync(kFullMask, ex, 0);
    u64 uu = sbase[0] + (wex & ((1ull << 21) - 1));
    u64 pp = sbase[1] + ((wex >> 21) & ((1ull << 21) - 1));
    u64 bb = sbase[2] + ((wex >> 42) & ((1ull << 21) - 1));
    const u32 lt = lanemask_lt();
    u64 mysum = 0;
    // quad symbols are 1..8 (qd = 0..7): lane v < 8 counts symbol v + 1 from three ballots of
    // its bits, and keeps the unit of its first occurrence
    u32 qn = 0, qf = 0xffffffffu;
    for (int r = 0; r < kItems; ++r) {
        const u32 e = wfirst + (u32)r * 32u + lane;
        u64 vi, idi;
        const u32 f = classify(e, vi, idi);
        const bool head = f & 1u;
        const bool patch = head && ((f >> 1) & 1u);
        const bool nblk = head && ((f >> 2) & 1u);
        const u32 hm = __ballot_sync(kFullMask, head), pm = __ballot_sync(kFullMask, patch),
                  bm = __ballot_sync(kFullMask, nblk);
        const u64 u = uu + __popc(hm & lt);
        const u32 sym = head ? (patch ? 0u : (u32)vi + 1u) : 0u;
        const u32 qsym = ((f >> 8) & 0xffu) + 1u;
        if (head) {
            out.rep_sym[u] = (u8)sym;
            if (out.rep_val) out.rep_val[u] = vi;
            if (!DIRECT) out.quad_sym[u] = (u8)qsym;
            if (patch) {
                out.patches[pp + __popc(pm & lt)] = vi;
                mysum += vi;
            }
            if (!DIRECT && nblk) {
                const u64 bi = bb + __popc(bm & lt);
                out.blk_id[bi] = idi;
                out.blk_unit[bi] = (u32)u;
            }
            if (rle) out.unit_pos[u] = (u32)(base + e);
        }
        hist_add_masked(mrep[w], hrep, frep, head, sym, (u32)u);
        if (!DIRECT) {
            const u32 qb = qsym - 1u;
            const u32 b0 = __ballot_sync(kFullMask, head && (qb & 1u)), b1 = __ballot_sync(kFullMask, head && (qb & 2u)),
                      b2 = __ballot_sync(kFullMask, head && (qb & 4u));
            const u32 mv = hm & ((lane & 1u) ? b0 : ~b0) & ((lane & 2u) ? b1 : ~b1) & ((lane & 4u) ? b2 : ~b2);
            if (lane < 8u && mv) {
                qn += (u32)__popc(mv);
                if (qf == 0xffffffffu) qf = (u32)(uu + (u32)__popc(hm & ((1u << (__ffs(mv) - 1)) - 1u)));
            }
        }
        uu += __popc(hm);
        pp += __popc(pm);
        bb += __popc(bm);
    }
    if (!DIRECT && lane < 8u && qn) {
        atomicAdd(&hquad[lane + 1], qn);
        atomicMin(&fquad[lane + 1], qf);
    }
    for (int d = 16; d > 0; d >>= 1) mysum += __shfl_xor_sync(kFullMask, mysum, d);
    if (lane_id() == 0) psum[tid >> 5] = mysum;
    __syncthreads();
    if (tid == 0) {
        u64 s = 0;
        for (int w = 0; w < kThreads / 32; ++w) s += psum[w];
        if (s) atomicAdd(&out.counters[3], s);
    }
    if (hrep[tid]) {
        atomicAdd(&out.hist_rep[tid], (u64)hrep[tid]);
        atomicMin(&out.first_rep[tid], frep[tid]);
    }
    if (!DIRECT && tid < 16 && hquad[tid]) {
        atomicAdd(&out.hist_quad[tid], (u64)hquad[tid]);
        atomicMin(&out.first_quad[tid], fquad[tid]);
    }
}

// -rle: count of each unit = distance to the next unit's first point.
__global__ void __launch_bounds__(kThreads) count_stats_kernel(const u32* __restrict__ unit_pos, u64 units, u64 n,
                                                               i32* __restrict__ counts, CountStats cs) {
    __shared__ u32 sh[kCountDense], sf[kCountDense];
    for (int i = threadIdx.x; i < kCountDense; i += kThreads) {
        sh[i] = 0;
        sf[i] = 0xffffffffu;
    }
    __syncthreads();
    const u64 stride = (u64)gridDim.x * kThreads;
    const u64 start = (u64)blockIdx.x * kThreads + (threadIdx.x & ~31u);
    for (u64 b0 = start; b0 < units; b0 += stride) {
        const u64 u = b0 + lane_id();
        const bool ok = u < units;
        u32 c = 0;
        if (ok) {
            if (unit_pos) {
                const u64 nxt = (u + 1 < units) ? (u64)unit_pos[u + 1] : n;
                c = (u32)(nxt - unit_pos[u]);
                counts[u] = (i32)c;
            } else {  // counts given (cell tables)
                c = (u32)counts[u];
            }
        }
        const bool dense = ok && c < (u32)kCountDense;
        hist_add(sh, sf, dense, c, (u32)u);
        if (ok && !dense) {
            const u32 slot = atomicAdd(cs.over_n, 1u);
            cs.over_val[slot] = c;
            cs.over_unit[slot] = (u32)u;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kCountDense; i += kThreads)
        if (sh[i]) {
            atomicAdd(&cs.hist[i], (u64)sh[i]);
            atomicMin(&cs.first[i], sf[i]);
        }
}

__global__ void __launch_bounds__(kThreads) block_deltas_kernel(const u64* __restrict__ blk_id,
                                                                const u32* __restrict__ blk_unit, u64 nb, u64 units,
                                                                u64* __restrict__ d_blk, u64* __restrict__ d_cnt,
                                                                u64* max2) {
    __shared__ u64 s0[kThreads / 32], s1[kThreads / 32];
    u64 m0 = 0, m1 = 0;
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 b = (u64)blockIdx.x * kThreads + threadIdx.x; b < nb; b += stride) {
        const u64 cb = ((b + 1 < nb) ? (u64)blk_unit[b + 1] : units) - blk_unit[b];
        u64 db, dc;
        if (b == 0) {
            db = blk_id[0];
            dc = cb;
        } else {
            const u64 cp = (u64)blk_unit[b] - blk_unit[b - 1];
            db = blk_id[b] - blk_id[b - 1];
            dc = cb - cp;  // wraps like the reference's in-place u64 differences
        }
        d_blk[b] = db;
        d_cnt[b] = dc;
        m0 = max(m0, db);
        m1 = max(m1, dc);
    }
    for (int d = 16; d > 0; d >>= 1) {
        m0 = max(m0, __shfl_xor_sync(kFullMask, m0, d));
        m1 = max(m1, __shfl_xor_sync(kFullMask, m1, d));
    }
    if (lane_id() == 0) {
        s0[threadIdx.x >> 5] = m0;
        s1[threadIdx.x >> 5] = m1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
            m0 = max(m0, s0[w]);
            m1 = max(m1, s1[w]);
        }
        m0 = max(m0, s0[0]);
        m1 = max(m1, s1[0]);
        atomicMax(&max2[0], m0);
        atomicMax(&max2[1], m1);
    }
}

// BitPacker: value b at bit b*width, LSB-first.  A warp packs 32 consecutive values (b0 a
// multiple of 32), which fill exactly `width` whole words of their own.  For widths 8..64,
// lane j builds words j and j + 32 (those below `width`) from the at most ceil(32 / width) + 1
// values each overlaps (shuffles) and stores them; narrower widths go through the warp's
// segmented-OR writer.  (Packing 32 values per thread into whole words, measured slower: 2.8
// -> 4.9 ms per 64M-point step, the per-thread 256-byte reads and width-word writes coalesce
// worse.)
__global__ void __launch_bounds__(kThreads) bitpack_kernel(const u64* __restrict__ vals, u64 n, int width,
                                                           u32* words) {
    const u64 stride = (u64)gridDim.x * kThreads;
    const u32 lane = lane_id();
    if (width >= 8 && width <= 64) {
        const u32 wu = (u32)width;
        const int K = (int)((32u + wu - 1u) / wu) + 1;
        const int halves = wu > 32u ? 2 : 1;
        u32 v0[2];
        int p0[2];
        for (int h = 0; h < 2; ++h) {
            const u32 m = lane + 32u * (u32)h;
            v0[h] = m < wu ? (32u * m) / wu : 0u;                // first value overlapping word m
            p0[h] = (int)(v0[h] * wu) - (int)(32u * m);         // its first bit relative to the word (<= 0)
        }
        const u64 vmask = wu >= 64u ? ~0ull : ((1ull << wu) - 1ull);
        const u64 total = n * (u64)wu;
        for (u64 b0 = (u64)blockIdx.x * kThreads + (threadIdx.x & ~31u); b0 < n; b0 += stride) {
            const u64 b = b0 + lane;
            const u64 x = b < n ? (vals[b] & vmask) : 0ull;
            for (int h = 0; h < halves; ++h) {
                const u32 m = lane + 32u * (u32)h;
                u32 word = 0;
                for (int k = 0; k < K; ++k) {
                    const u32 v = v0[h] + (u32)k;
                    const u64 xv = __shfl_sync(kFullMask, x, (int)(v & 31u));
                    const int pos = p0[h] + k * (int)wu;
                    if (m < wu && v < 32u && pos < 32) word |= pos >= 0 ? (u32)(xv << pos) : (u32)(xv >> (-pos));
                }
                const u64 wi = (b0 >> 5) * (u64)wu + m;
                if (m < wu && wi * 32u < total) words[wi] = word;
            }
        }
        return;
    }
    for (u64 b0 = (u64)blockIdx.x * kThreads + (threadIdx.x & ~31u); b0 < n; b0 += stride) {
        const u64 b = b0 + lane;
        const bool ok = b < n;
        warp_write_lsb(words, b * (u64)width, ok ? vals[b] : 0ull, ok ? (u32)width : 0u);
    }
}

// Shared skeleton of the chained-scan encoders: stage a tile of inputs, give every element
// its bit length, scan, look back, write.
template <typename T>
__device__ __forceinline__ u32 stage_tile(const T* __restrict__ in, u64 n, T* s, u32* slot, u32* tile_counter,
                                          u32& tile, u64& base) {
    tile = claim_tile(tile_counter, slot);
    base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, n - base);
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + threadIdx.x;
        if (e < cnt) s[e] = in[base + e];
    }
    __syncthreads();
    return cnt;
}

__device__ __forceinline__ u64 tile_bit_base(LookBackState lb, u32 tile, u64 tot, u64* sbase,
                                             unsigned long long* total_bits, u32* err) {
    if (threadIdx.x < 32) {
        LookBack64 l{lb.flag, lb.agg, lb.inc};
        const u64 before = warp_lookback_add(l, tile, tot, err);
        if (threadIdx.x == 0) {
            *sbase = before;
            if (tile == gridDim.x - 1) *total_bits = before + tot;
        }
    }
    __syncthreads();
    return *sbase;
}

// Thread t codes the tile's values [16 t, 16 t + 16) as one run of consecutive codewords:
// its values are read straight from global memory (two per 16-byte load) and kept in
// registers for the length sum and the writes; the run's bits leave a word at a time
// (LsbRun), so a thread makes about one memory operation per 32 bits of output.
__global__ void __launch_bounds__(kThreads) gr_encode_kernel(const u64* __restrict__ vals, u64 n, int k, u32* words,
                                                             u64 cap_bits, LookBackState lb, u32* tile_counter,
                                                             unsigned long long* total_bits, u32* err) {
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase;
    const u32 tile = claim_tile(tile_counter, &slot);
    const u64 base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, n - base);
    const u32 e0 = threadIdx.x * kItems;
    u64 v[kItems];
    const bool vec = e0 + kItems <= cnt && ((reinterpret_cast<uintptr_t>(vals + base + e0) & 15u) == 0);
    if (vec) {
#pragma unroll
        for (int i = 0; i < kItems; i += 2) {
            const ulonglong2 p = __ldg(reinterpret_cast<const ulonglong2*>(vals + base + e0 + i));
            v[i] = p.x;
            v[i + 1] = p.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < kItems; ++i) v[i] = e0 + i < cnt ? __ldg(vals + base + e0 + i) : 0ull;
    }
    u64 sum = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (e0 + i < cnt) sum += (v[i] >> k) + 1u + (u64)k;
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(sum, 0ull, AddOp{}, scratch, tot);
    const u64 pos = tile_bit_base(lb, tile, tot, &sbase, total_bits, err) + ex;
    if (pos + sum > cap_bits) {  // output bound (never reached with valid sizes)
        if (sum) atomicOr(err, kErrOverflow);
        return;
    }
    const u64 mask = k ? ((1ull << k) - 1) : 0ull;
    LsbRun run;
    run.begin(words, pos);
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (e0 + i >= cnt) continue;
        const u64 q = v[i] >> k;
        const u64 r = v[i] & mask;
        if (q + 1u + (u64)k <= 32u) {  // unary part, terminating zero and remainder in one piece
            run.put32((u32)((q ? ((1ull << q) - 1) : 0ull) | (r << (q + 1))), (u32)(q + 1u + (u64)k));
        } else {
            run.ones(q);
            run.put32(0u, 1u);
            run.put(r, (u32)k);
        }
    }
    run.end();
}

__global__ void __launch_bounds__(kThreads) huff_encode_u8_kernel(const u8* __restrict__ sym, u64 n,
                                                                  const ByteCodes* __restrict__ codes, u32* words,
                                                                  u64 cap_bits, LookBackState lb, u32* tile_counter,
                                                                  unsigned long long* total_bits, u32* err) {
    __shared__ u8 ss[kTile];
    __shared__ u32 cbits[256];
    __shared__ u8 clen[256];
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase;
    cbits[threadIdx.x] = codes->bits[threadIdx.x];
    clen[threadIdx.x] = codes->len[threadIdx.x];
    u32 tile;
    u64 base;
    const u32 cnt = stage_tile(sym, n, ss, &slot, tile_counter, tile, base);
    const u32 e0 = threadIdx.x * kItems;
    u64 sum = 0;
#pragma unroll
    for (int i = 0; i < kItems; ++i)
        if (e0 + i < cnt) sum += clen[ss[e0 + i]];
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(sum, 0ull, AddOp{}, scratch, tot);
    u64 pos = tile_bit_base(lb, tile, tot, &sbase, total_bits, err) + ex;
    if (pos + sum > cap_bits) {  // output bound (never reached with valid sizes)
        if (sum) atomicOr(err, kErrOverflow);
        return;
    }
    MsbRun run;
    run.begin(words, pos);
#pragma unroll 4
    for (int i = 0; i < kItems; ++i) {
        if (e0 + i >= cnt) break;
        const u32 s = ss[e0 + i];
        const u32 len = clen[s];
        // Codes longer than 32 bits are the 32-bit value zero-extended (huffman_encoder.hpp:251).
        if (len > 32u) {
            run.zeros(len - 32u);
            run.put32(cbits[s], 32u);
        } else {
            run.put32(cbits[s], len);
        }
    }
    run.end();
}

// A prefix code whose codewords all have one length L (1..24 bits): symbol i occupies stream
// bits [i L, (i + 1) L), so no scan is needed.  Thread g codes symbols [32 g, 32 g + 32), whose
// 32 L bits fill exactly words [g L, g L + L), MSB-first and stored byte-swapped as MsbRun
// stores them; whole words, no atomics.  Symbols index code_bits (counts: the dense table).
template <typename T>
__global__ void __launch_bounds__(kThreads) fixed_encode_kernel(const T* __restrict__ sym, u64 n,
                                                                const u32* __restrict__ code_bits, int len,
                                                                u32* __restrict__ words,
                                                                unsigned long long* total_bits) {
    const u64 g = (u64)blockIdx.x * kThreads + threadIdx.x;
    const u64 total = n * (u64)len;
    if (g == 0) *total_bits = total;
    const u64 s0 = g * 32u;
    if (s0 >= n) return;
    const u32 mask = (1u << len) - 1u;
    u64 acc = 0, w = g * (u64)len;
    u32 nb = 0;
#pragma unroll 4
    for (int i = 0; i < 32; ++i) {
        const u64 idx = s0 + (u64)i;
        const u32 c = idx < n ? (__ldg(&code_bits[(u32)sym[idx]]) & mask) : 0u;
        acc = (acc << len) | c;
        nb += (u32)len;
        if (nb >= 32u) {
            nb -= 32u;
            if (w * 32u < total) words[w] = __byte_perm((u32)(acc >> nb), 0, 0x0123);
            ++w;
            acc &= nb ? ((1ull << nb) - 1ull) : 0ull;
        }
    }
}

__device__ __forceinline__ u32 rev_low(u64 v, int k) { return k ? (__brev((u32)v) >> (32 - k)) : 0u; }

__global__ void __launch_bounds__(kThreads) count_encode_kernel(const i32* __restrict__ counts, u64 n, int eg_k,
                                                                const u32* __restrict__ dense_bits,
                                                                const u8* __restrict__ dense_len,
                                                                const u32* __restrict__ sparse_val,
                                                                const u32* __restrict__ sparse_bits,
                                                                const u8* __restrict__ sparse_len, u32 sparse_n,
                                                                u32* words, u64 cap_bits, LookBackState lb,
                                                                u32* tile_counter,
                                                                unsigned long long* total_bits, u32* err) {
    __shared__ i32 sc[kTile];
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase;
    u32 tile;
    u64 base;
    const u32 cnt = stage_tile(counts, n, sc, &slot, tile_counter, tile, base);
    const u32 e0 = threadIdx.x * kItems;
    // code of one count: (length, value bits, bit offset of the value inside the code)
    auto code = [&](i32 c, u32& len, u64& val, u32& nb) {
        if (eg_k >= 0) {
            const long long s = c;
            const u64 z = ((u64)s << 1) ^ (u64)(s >> 63);
            const u64 n1 = (z >> eg_k) + 1u;
            const u32 lz = bitlen64(n1) - 1u;
            len = 2u * lz + 1u + (u32)eg_k;
            nb = lz + 1u + (u32)eg_k;
            val = (n1 << eg_k) | rev_low(z, eg_k);
        } else {
            const u32 uc = (u32)c;
            u32 bits = 0, l = 0;
            if (uc < (u32)kCountDense) {
                bits = dense_bits[uc];
                l = dense_len[uc];
            } else {
                u32 lo = 0, hi = sparse_n;
                while (lo < hi) {
                    const u32 mid = (lo + hi) >> 1;
                    if (sparse_val[mid] < uc) lo = mid + 1; else hi = mid;
                }
                if (lo < sparse_n && sparse_val[lo] == uc) {
                    bits = sparse_bits[lo];
                    l = sparse_len[lo];
                } else {
                    atomicOr(err, kErrOverflow);
                }
            }
            len = l;
            nb = l > 32u ? 32u : l;
            val = bits;
        }
    };
    u64 sum = 0;
    for (int i = 0; i < kItems; ++i)
        if (e0 + i < cnt) {
            u32 len, nb;
            u64 val;
            code(sc[e0 + i], len, val, nb);
            sum += len;
        }
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(sum, 0ull, AddOp{}, scratch, tot);
    u64 pos = tile_bit_base(lb, tile, tot, &sbase, total_bits, err) + ex;
    if (pos + sum > cap_bits) {  // output bound (never reached with valid sizes)
        if (sum) atomicOr(err, kErrOverflow);
        return;
    }
    MsbRun run;
    run.begin(words, pos);
    for (int i = 0; i < kItems; ++i) {
        if (e0 + i >= cnt) break;
        u32 len, nb;
        u64 val;
        code(sc[e0 + i], len, val, nb);
        run.zeros(len - nb);  // exp-Golomb's leading zeros, or a long Huffman code's extension
        run.put(val, nb);
    }
    run.end();
}

inline int persistent_grid(u64 n) {
    u64 want = (n + kThreads - 1) / kThreads;
    if (want < 1) want = 1;
    return (int)(want < 148ull * 8ull ? want : 148ull * 8ull);
}

}  // namespace

void launch_units_block(const unsigned long long* keys, uint64_t n, int rle, BlockKeyParams kp, UnitOutputs out,
                        LookBackState lb, uint32_t* tile_counter, uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    units_kernel<false><<<tiles, kThreads, 0, st>>>(keys, n, rle, kp, DirectKeyParams{}, out, lb, tile_counter, err);
}
void launch_units_direct(const unsigned long long* keys, uint64_t n, int rle, DirectKeyParams kp, UnitOutputs out,
                         LookBackState lb, uint32_t* tile_counter, uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    units_kernel<true><<<tiles, kThreads, 0, st>>>(keys, n, rle, BlockKeyParams{}, kp, out, lb, tile_counter, err);
}
void launch_count_stats(const uint32_t* unit_pos, uint64_t units, uint64_t n, int32_t* counts, CountStats cs,
                        cudaStream_t st) {
    count_stats_kernel<<<persistent_grid(units), kThreads, 0, st>>>(unit_pos, units, n, counts, cs);
}
void launch_block_deltas(const unsigned long long* blk_id, const uint32_t* blk_unit, uint64_t nblocks, uint64_t units,
                         unsigned long long* d_blk, unsigned long long* d_cnt, unsigned long long* max2,
                         cudaStream_t st) {
    block_deltas_kernel<<<persistent_grid(nblocks), kThreads, 0, st>>>(blk_id, blk_unit, nblocks, units, d_blk, d_cnt,
                                                                       max2);
}
void launch_bitpack(const unsigned long long* vals, uint64_t n, int width, uint32_t* words, cudaStream_t st) {
    bitpack_kernel<<<persistent_grid(n), kThreads, 0, st>>>(vals, n, width, words);
}
void launch_gr_encode(const unsigned long long* vals, uint64_t n, int k, uint32_t* words, uint64_t cap_bits,
                      LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits, uint32_t* err,
                      cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    gr_encode_kernel<<<tiles, kThreads, 0, st>>>(vals, n, k, words, cap_bits, lb, tile_counter, total_bits, err);
}
void launch_fixed_encode_u8(const uint8_t* sym, uint64_t n, const uint32_t* code_bits, int len, uint32_t* words,
                            unsigned long long* total_bits, cudaStream_t st) {
    const u64 threads = (n + 31) / 32;
    const unsigned blocks = (unsigned)((threads + kThreads - 1) / kThreads);
    fixed_encode_kernel<u8><<<blocks ? blocks : 1, kThreads, 0, st>>>(sym, n, code_bits, len, words, total_bits);
}
void launch_fixed_encode_i32(const int32_t* sym, uint64_t n, const uint32_t* code_bits, int len, uint32_t* words,
                             unsigned long long* total_bits, cudaStream_t st) {
    const u64 threads = (n + 31) / 32;
    const unsigned blocks = (unsigned)((threads + kThreads - 1) / kThreads);
    fixed_encode_kernel<i32><<<blocks ? blocks : 1, kThreads, 0, st>>>(sym, n, code_bits, len, words, total_bits);
}
void launch_huff_encode_u8(const uint8_t* sym, uint64_t n, const ByteCodes* codes, uint32_t* words,
                           uint64_t cap_bits, LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits,
                           uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    huff_encode_u8_kernel<<<tiles, kThreads, 0, st>>>(sym, n, codes, words, cap_bits, lb, tile_counter, total_bits,
                                                      err);
}
void launch_count_encode(const int32_t* counts, uint64_t n, int eg_k, const uint32_t* dense_bits,
                         const uint8_t* dense_len, const uint32_t* sparse_val, const uint32_t* sparse_bits,
                         const uint8_t* sparse_len, uint32_t sparse_n, uint32_t* words, uint64_t cap_bits,
                         LookBackState lb, uint32_t* tile_counter, unsigned long long* total_bits, uint32_t* err,
                         cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    count_encode_kernel<<<tiles, kThreads, 0, st>>>(counts, n, eg_k, dense_bits, dense_len, sparse_val, sparse_bits,
                                                    sparse_len, sparse_n, words, cap_bits, lb, tile_counter,
                                                    total_bits, err);
}

}  // namespace dev
}  // namespace xnyz
