// Decompress-side kernels.
//
//   block_streams  BitPacker<uint64_t>::unpack (encoder/bitpacking_encoder.hpp:53-80) of the
//                  block-id and block-count deltas fused with their prefix sums
//                  (block_decompressor.hpp:159-161, u64, wrapping) and the block-start marks
//   (the entropy-coded streams are decoded in k_stream_decode.cu)
//   recover_units  recover_from_lcp_meta (block_quantizer.hpp:154-207) fused with the PFor
//                  decode, the direct-mode SFC prefix sum (block_decompressor.hpp:86-102), the
//                  -rle expansion (block_decompressor_rle.hpp:182-187), recover and unshift.
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;
static_assert(kTile == kScanTile, "tile size");

// x / d for an invariant divisor (U64Div, kernels.h)
__device__ __forceinline__ u64 udiv(u64 x, const U64Div& d) {
    const u64 t = __umul64hi(d.m, x);
    return (t + ((x - t) >> d.sh1)) >> d.sh2;
}

// ------------------------------------------------------------- block streams -----------
// The -normal/-rle block streams of block mode in one pass (block_decompressor.hpp:111-161):
// bit-unpack the block-id deltas and block-count deltas, inclusive prefix sums of both
// (u64, wrapping), the exclusive prefix of the counts (first unit of each block), and the
// per-unit block-start marks of recover_from_lcp_meta (block_quantizer.hpp:167-176).
// The count channel carries (sum of deltas, blocks, sum of counts) so that the prefix of the
// counts and the prefix of their prefix come out of one chained scan:
//   (A1, N1, B1) then (A2, N2, B2) = (A1 + A2, N1 + N2, B1 + B2 + N2 * A1).
struct Tri {
    u64 a, n, b;
};
struct TriOp {
    __device__ __forceinline__ Tri operator()(Tri x, Tri y) const { return Tri{x.a + y.a, x.n + y.n, x.b + y.b + y.n * x.a}; }
};
struct LoadTri {
    __device__ __forceinline__ Tri operator()(const Tri* p) const {
        return Tri{ld_volatile(&p->a), ld_volatile(&p->n), ld_volatile(&p->b)};
    }
};
struct StoreTri {
    __device__ __forceinline__ void operator()(Tri* p, Tri v) const {
        st_volatile(&p->a, v.a);
        st_volatile(&p->n, v.n);
        st_volatile(&p->b, v.b);
    }
};
// found by argument-dependent lookup from warp_lookback
__device__ __forceinline__ Tri shfl_down_t(Tri v, int d) {
    return Tri{__shfl_down_sync(kFullMask, v.a, d), __shfl_down_sync(kFullMask, v.n, d),
               __shfl_down_sync(kFullMask, v.b, d)};
}
__device__ __forceinline__ Tri shfl_t(Tri v, int l) {
    return Tri{__shfl_sync(kFullMask, v.a, l), __shfl_sync(kFullMask, v.n, l), __shfl_sync(kFullMask, v.b, l)};
}

__global__ void __launch_bounds__(kThreads) block_streams_kernel(const u32* __restrict__ wb, u64 bb, int width_b,
                                                                 const u32* __restrict__ wc, u64 bc, int width_c,
                                                                 u64 nb, u64 units, u64* __restrict__ blk_out,
                                                                 u8* __restrict__ is_start, u32* __restrict__ start_block,
                                                                 LookBackState lb, u32* tile_counter,
                                                                 unsigned long long* count_total, u32* err) {
    constexpr int kWarps = kThreads / 32;
    __shared__ u32 slot;
    __shared__ u64 wsb[kWarps + 1];
    __shared__ Tri wtc[kWarps + 1];
    __shared__ u64 base_b;
    __shared__ Tri base_c;
    const u32 tile = claim_tile(tile_counter, &slot);
    const u32 ntiles = gridDim.x;
    const int tid = threadIdx.x;
    const int w = tid >> 5;
    const u32 lane = lane_id();
    // warp w owns blocks [512 w, 512 w + 512) of the tile, 32 consecutive blocks per round
    const u64 wfirst = (u64)tile * kTile + (u64)w * (32u * kItems);
    const u64 mb = width_b >= 64 ? ~0ull : ((1ull << width_b) - 1), mc = width_c >= 64 ? ~0ull : ((1ull << width_c) - 1);
    auto delta_b = [&](u64 j) { return width_b ? (peek_lsb64(wb, bb + j * (u64)width_b) & mb) : 0ull; };
    auto delta_c = [&](u64 j) { return width_c ? (peek_lsb64(wc, bc + j * (u64)width_c) & mc) : 0ull; };

    // Running values along the warp's blocks: blk (block id), cnt (block count = inclusive
    // sum of the count deltas), start (first unit of the block = exclusive sum of the
    // counts).  The warp's aggregates need no scans (below); the pass from the true carries
    // writes the outputs.
    auto pass = [&](u64& blk, u64& cnt, u64& start) {
        for (int r = 0; r < kItems; ++r) {
            const u64 j = wfirst + (u64)r * 32u + lane;
            const bool valid = j < nb;
            const u64 db = valid ? delta_b(j) : 0ull, dc = valid ? delta_c(j) : 0ull;
            const u64 bj = blk + warp_incl_add(db);
            const u64 cj = cnt + warp_incl_add(dc);
            const u64 vc = valid ? cj : 0ull;
            const u64 ci = warp_incl_add(vc);
            const u64 sj = start + ci - vc;
            blk = __shfl_sync(kFullMask, bj, 31);
            cnt = __shfl_sync(kFullMask, cj, 31);
            start += __shfl_sync(kFullMask, ci, 31);
            if (valid) {
                blk_out[j] = bj;
                if (cj > 0 && sj < units) {  // non-empty block (the reference skips empty ones)
                    is_start[sj] = 1;
                    start_block[sj] = (u32)j;
                }
            }
        }
    };
    {
        // From zero carries the warp ends at blk = sum of db, cnt = sum of dc, and start = the
        // sum of its m blocks' counts c_j = dc_0 + .. + dc_j, which is the sum over i of
        // dc_i * (m - i) (u64, wrapping like the running sums).
        const u64 wbeg = wfirst < nb ? wfirst : nb;
        const u64 nvalid = (nb - wbeg) < 32u * kItems ? nb - wbeg : 32u * kItems;
        u64 sb = 0, sc = 0, sw = 0;
        for (int r = 0; r < kItems; ++r) {
            const u64 i = (u64)r * 32u + lane;
            if (wfirst + i < nb) {
                const u64 dc = delta_c(wfirst + i);
                sb += delta_b(wfirst + i);
                sc += dc;
                sw += dc * (nvalid - i);
            }
        }
        sb = warp_sum(sb);
        sc = warp_sum(sc);
        sw = warp_sum(sw);
        if (lane == 0) {
            wsb[w] = sb;
            wtc[w] = Tri{sc, nvalid, sw};
        }
    }
    __syncthreads();
    if (tid == 0) {
        warps_exclusive<kWarps>(wsb, 0ull, AddOp{});
        warps_exclusive<kWarps>(wtc, Tri{0, 0, 0}, TriOp{});
    }
    __syncthreads();
    if (tid < 32) {
        LookBack64 l{lb.flag, lb.agg, lb.inc};
        const u64 r = warp_lookback_add(l, tile, wsb[kWarps], err);
        if (tid == 0) base_b = r;
    } else if (tid < 64) {
        Tri* ag = reinterpret_cast<Tri*>(lb.agg + ntiles);
        Tri* in = reinterpret_cast<Tri*>(lb.inc + ntiles);
        const Tri r = warp_lookback(lb.flag + ntiles, ag, in, tile, wtc[kWarps], Tri{0, 0, 0}, TriOp{}, LoadTri{},
                                    StoreTri{}, err);
        if (tid == 32) {
            base_c = r;
            if (tile == ntiles - 1) *count_total = TriOp{}(r, wtc[kWarps]).b;
        }
    }
    __syncthreads();
    const Tri pre = TriOp{}(base_c, wtc[w]);
    u64 blk = base_b + wsb[w], cnt = pre.a, start = pre.b;
    pass(blk, cnt, start);
}

// ---------------------------------------------------------------- helpers --------------
__global__ void fill_u32_kernel(u32* p, u64 n, u32 v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void fill_u8_kernel(u8* p, u64 n, u8 v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void __launch_bounds__(kThreads) count_total_kernel(const i32* __restrict__ c, u64 n,
                                                               unsigned long long* total) {
    u64 s = 0;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += (u64)gridDim.x * kThreads)
        s += (u64)max(c[i], 0);
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(kFullMask, s, d);
    if (lane_id() == 0 && s) atomicAdd(total, s);
}

// ------------------------------------------------------------- recover units -------------
struct RecoverArgs {
    const u8* rep_sym;
    const u64* rep_patch;
    u64 npatch;
    const u8* quad_sym;
    const u8* is_start;
    const u32* start_block;
    const u64* blk_ids;
    u64 nblocks;
    const i32* counts;
    const u64* rep_val;
    u64 units;
    u64 nout;
    RecoverParams rp;
    const u8* hinv;
    u32* flag;   // [5][ntiles]
    u64* agg;    // [5][ntiles][2]
    u64* inc;    // [5][ntiles][2]
    u32* tile_counter;
    float* out;
    u32* err;
};

// Quad index step of a packed quad symbol (see recover_units_kernel): q - 1 modulo 8, 0 for
// the patch symbol 0.
__device__ __forceinline__ u32 quad_step(u32 sq) { return (sq & 8u) ? 0u : ((sq + 7u) & 7u); }

// Warp w owns units [512 w, 512 w + 512) of the tile and takes them 32 at a time, one per
// lane: staged symbols are read without bank conflicts, patches, counts and block starts
// are read coalesced, and the points of a round are written to consecutive addresses.
// Phase 1 counts each warp's zero symbols in shared memory (the tile's first patch index
// then comes from a chained scan that every tile publishes right after staging); phase 2
// reads the patches and counts once, keeps each unit's repos value (or SFC delta) and count
// in shared memory, and folds the warp's counts, quad / block / repos segments (or SFC
// sums); the block combines the warps, one round of chained scans combines the tiles, and
// the final pass rebuilds every running value with warp scans from its warp's starting
// carry.  A tile holding a value of 2^32 or more or a count of 2^16 or more re-reads them
// in the final pass instead (block mode: never for a stream the encoder wrote, whose repos
// values are 18-bit codes; direct mode: the tile of a cloud's first SFC code, for example).
// With every value below 2^26 as well, the rounds' prefix sums run in 32 bits.
template <bool DIRECT>
__global__ void __launch_bounds__(kThreads, 6) recover_units_kernel(RecoverArgs a) {
    constexpr int kWarps = kThreads / 32;
    __shared__ u8 srep[kTile];
    // block mode: quad symbol q's low 3 bits | 8 (q == 0) | 16 (q == 1) | 32 (block start);
    // the quad index is only used modulo 8, so its running sums need nothing more
    __shared__ u8 squad[DIRECT ? 1 : kTile];
    __shared__ u32 sval[kTile];
    __shared__ u16 scnt[kTile];
    __shared__ u32 slot, wide;
    __shared__ u64 wz[kWarps + 1], wc[kWarps + 1], wd[kWarps + 1];
    __shared__ Seg wq[kWarps + 1], wb[kWarps + 1], wr[kWarps + 1];
    __shared__ u64 base_zero, base_count, base_sfc;
    __shared__ Seg base_quad, base_blk, base_rep;
    __shared__ u8 htab[256];

    const u32 tile = claim_tile(a.tile_counter, &slot);
    const u32 ntiles = gridDim.x;
    const u64 base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, a.units - base);
    const int tid = threadIdx.x;
    const int w = tid >> 5;
    const u32 lane = lane_id();
    const u32 lt = lanemask_lt();
    const bool has_val = a.rep_val != nullptr;
    for (int i = tid; i < 256; i += kThreads) htab[i] = a.hinv ? a.hinv[i] : 0;
    if (tid == 0) wide = 0;
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + tid;
        if (e < cnt) {
            srep[e] = has_val ? (u8)1 : a.rep_sym[base + e];
            if (!DIRECT) {
                const u32 qs = a.quad_sym[base + e];
                squad[e] = (u8)((qs & 7u) | (qs == 0 ? 8u : 0u) | (qs == 1 ? 16u : 0u) |
                                (a.is_start[base + e] ? 32u : 0u));
            }
        }
    }
    __syncthreads();
    const bool rle = a.rp.rle != 0;
    const u32 wfirst = (u32)w * (32u * kItems);
    SegOp op;

    // repos value of unit e; zc: index of the warp's next patch (advanced on symbol 0).
    // Called by all lanes (it votes).
    auto rep_value = [&](u32 e, bool valid, u64& zc) -> u64 {
        const u32 sym = valid ? srep[e] : 1u;
        const u32 zb = __ballot_sync(kFullMask, valid && !has_val && sym == 0u);
        const u64 z = zc + __popc(zb & lt);
        zc += __popc(zb);
        if (!valid) return 0;
        if (has_val) return a.rep_val[base + e];
        if (sym) return sym - 1u;
        if (z < a.npatch) return a.rep_patch[z];
        atomicOr(a.err, kErrBadStream);
        return 0;
    };

    // ---- phase 1: zero symbols per warp, chained into the tile's first patch index ----
    if (!has_val) {
        u64 z = 0;
        for (int r = 0; r < kItems; ++r) {
            const u32 e = wfirst + (u32)r * 32u + lane;
            z += __popc(__ballot_sync(kFullMask, e < cnt && srep[e] == 0));
        }
        if (lane == 0) wz[w] = z;
        __syncthreads();
        if (tid == 0) warps_exclusive<kThreads / 32>(wz, 0ull, AddOp{});
        __syncthreads();
        if (w == 0) {
            LookBack64 l{a.flag, a.agg, a.inc};
            const u64 r = warp_lookback_add(l, tile, wz[kWarps], a.err);
            if (tid == 0) base_zero = r;
        }
    } else if (tid < kWarps) {
        wz[tid] = 0;
        if (tid == 0) base_zero = 0;
    }
    __syncthreads();

    // ---- phase 2: values and counts kept; counts, quad, block, repos segments per warp ----
    {
        u64 zc = base_zero + wz[w];
        u64 c = 0, d = 0, bc = 0, rc = 0;
        u32 qc = 0;
        bool any_head = false, any_rhead = false, big = false, w26 = false;
        for (int r = 0; r < kItems; ++r) {
            const u32 e = wfirst + (u32)r * 32u + lane;
            const bool valid = e < cnt;
            const u64 v = rep_value(e, valid, zc);
            const u64 k = rle && valid ? (u64)max(a.counts[base + e], 0) : 0ull;
            c += k;
            if (valid) {
                sval[e] = (u32)v;
                scnt[e] = (u16)k;
                big |= (v >> 32) != 0 || (k >> 16) != 0;
                w26 |= (v >> 26) != 0;
            }
            if (DIRECT) {
                d += v;
            } else {
                const u32 sq = valid ? squad[e] : 16u;
                const bool st = (sq & 32u) != 0;
                const u32 hm = __ballot_sync(kFullMask, st);
                qc = __shfl_sync(kFullMask, warp_seg_incl<u32>(hm, quad_step(sq), qc), 31);
                const u32 bv = st ? a.start_block[base + e] : 0u;
                const u32 last = __shfl_sync(kFullMask, bv, hm ? 31 - __clz(hm) : 0);
                if (hm) bc = last;
                any_head |= hm != 0;
                const u32 hr = __ballot_sync(kFullMask, valid && (st || (sq & 16u) == 0));
                rc = __shfl_sync(kFullMask, warp_seg_incl<u64>(hr, v, rc), 31);
                any_rhead |= hr != 0;
            }
        }
        c = warp_sum(c);
        if (DIRECT) d = warp_sum(d);
        const bool anybig = __any_sync(kFullMask, big), any26 = __any_sync(kFullMask, w26);
        if (lane == 0 && (anybig || any26)) atomicOr(&wide, (anybig ? 1u : 0u) | (any26 ? 2u : 0u));
        if (lane == 0) {
            wc[w] = c;
            wd[w] = d;
            wq[w] = Seg{any_head ? 1ull : 0ull, (u64)qc};
            wb[w] = Seg{any_head ? 1ull : 0ull, bc};
            wr[w] = Seg{any_rhead ? 1ull : 0ull, rc};
        }
    }
    __syncthreads();
    if (tid == 0) {
        warps_exclusive<kThreads / 32>(wc, 0ull, AddOp{});
        if (DIRECT) {
            warps_exclusive<kThreads / 32>(wd, 0ull, AddOp{});
        } else {
            warps_exclusive<kThreads / 32>(wq, Seg{0, 0}, op);
            warps_exclusive<kThreads / 32>(wb, Seg{0, 0}, op);
            warps_exclusive<kThreads / 32>(wr, Seg{0, 0}, op);
        }
    }
    __syncthreads();
    // one warp per chained scan
    if (w == 0) {
        if (DIRECT) {
            LookBack64 l{a.flag + 4 * ntiles, a.agg + 8ull * ntiles, a.inc + 8ull * ntiles};
            const u64 r = warp_lookback_add(l, tile, wd[kWarps], a.err);
            if (tid == 0) base_sfc = r;
        } else {
            Seg* ag = reinterpret_cast<Seg*>(a.agg + 8ull * ntiles);
            Seg* in = reinterpret_cast<Seg*>(a.inc + 8ull * ntiles);
            const Seg r = warp_lookback(a.flag + 4 * ntiles, ag, in, tile, wr[kWarps], Seg{0, 0}, SegOp{}, LoadSeg{},
                                        StoreSeg{}, a.err);
            if (tid == 0) base_rep = r;
        }
    } else if (w == 1 && rle) {
        LookBack64 l{a.flag + ntiles, a.agg + 2ull * ntiles, a.inc + 2ull * ntiles};
        const u64 r = warp_lookback_add(l, tile, wc[kWarps], a.err);
        if (tid == 32) base_count = r;
    } else if (w == 2 && !DIRECT) {
        Seg* ag = reinterpret_cast<Seg*>(a.agg + 4ull * ntiles);
        Seg* in = reinterpret_cast<Seg*>(a.inc + 4ull * ntiles);
        const Seg r = warp_lookback(a.flag + 2 * ntiles, ag, in, tile, wq[kWarps], Seg{0, 0}, SegOp{}, LoadSeg{},
                                    StoreSeg{}, a.err);
        if (tid == 64) base_quad = r;
    } else if (w == 3 && !DIRECT) {
        Seg* ag = reinterpret_cast<Seg*>(a.agg + 6ull * ntiles);
        Seg* in = reinterpret_cast<Seg*>(a.inc + 6ull * ntiles);
        const Seg r = warp_lookback(a.flag + 3 * ntiles, ag, in, tile, wb[kWarps], Seg{0, 0}, SegOp{}, LoadSeg{},
                                    StoreSeg{}, a.err);
        if (tid == 96) base_blk = r;
    }
    if (!rle && tid == 0) base_count = 0;
    __syncthreads();

    // ---- final: coordinates, recover, unshift, expand ----
    const QuantParams q = a.rp.q;
    // block-uniform: values and counts kept in shared memory; and, with every value below 2^26
    // and every count below 2^16, the round's prefix sums fit 32 bits
    const bool kept = (wide & 1u) == 0;
    const bool narrow = wide == 0;
    u64 zc = base_zero + wz[w];
    u64 oc = base_count + wc[w];  // -rle: output position of the warp's first point
    u64 scar = DIRECT ? base_sfc + wd[w] : 0ull;
    u32 qcar = DIRECT ? 0u : (u32)op(base_quad, wq[w]).sum;
    u64 rcar = DIRECT ? 0ull : op(base_rep, wr[w]).sum;
    // corner of the block of the warp's current unit ((blk % nx) * 128, (blk / nx % ny) * 128,
    // (blk / nx / ny) * 128 in u64 arithmetic, kept modulo 2^32 like the cell coordinates they
    // are added to): computed where a block starts, carried to the units after it
    u32 pcx = 0, pcy = 0, pcz = 0;
    auto corner = [&](u64 b, u32& x, u32& y, u32& z) {
        const u64 blk = b < a.nblocks ? a.blk_ids[b] : 0ull;
        const u64 q1 = udiv(blk, a.rp.div_nx), q2 = udiv(q1, a.rp.div_ny);
        x = (u32)((blk - q1 * a.rp.nx) * 128);
        y = (u32)((q1 - q2 * a.rp.ny) * 128);
        z = (u32)(q2 * 128);
    };
    if (!DIRECT) corner(op(base_blk, wb[w]).sum, pcx, pcy, pcz);
    for (int r = 0; r < kItems; ++r) {
        const u32 e = wfirst + (u32)r * 32u + lane;
        const bool valid = e < cnt;
        const u64 rv = kept ? (valid ? (u64)sval[e] : 0ull) : rep_value(e, valid, zc);
        i32 cx = 0, cy = 0, cz = 0;
        if (DIRECT) {
            const u64 sfc = scar + (narrow ? (u64)warp_incl_add((u32)rv) : warp_incl_add(rv));
            scar = __shfl_sync(kFullMask, sfc, 31);
            u32 gx, gy, gz;
            if (a.rp.hilbert) {
                hilbert_xyz(htab, sfc, a.rp.bits, 0u, gx, gy, gz);
            } else {
                gx = gather3(sfc);
                gy = gather3(sfc >> 1);
                gz = gather3(sfc >> 2);
            }
            cx = (i32)gx;
            cy = (i32)gy;
            cz = (i32)gz;
        } else {
            const u32 sq = valid ? squad[e] : 16u;
            const bool st = (sq & 32u) != 0;
            const u32 hm = __ballot_sync(kFullMask, st);
            const u32 quadj = warp_seg_incl<u32>(hm, quad_step(sq), qcar);
            qcar = __shfl_sync(kFullMask, quadj, 31);
            u32 sx = 0, sy = 0, sz = 0;
            if (st) corner(a.start_block[base + e], sx, sy, sz);
            const u32 le = hm & (lt | (1u << lane));
            const int src = le ? 31 - __clz(le) : 0;
            sx = __shfl_sync(kFullMask, sx, src);
            sy = __shfl_sync(kFullMask, sy, src);
            sz = __shfl_sync(kFullMask, sz, src);
            const u32 pbx = le ? sx : pcx, pby = le ? sy : pcy, pbz = le ? sz : pcz;
            pcx = __shfl_sync(kFullMask, pbx, 31);
            pcy = __shfl_sync(kFullMask, pby, 31);
            pcz = __shfl_sync(kFullMask, pbz, 31);
            const u32 hr = __ballot_sync(kFullMask, valid && (st || (sq & 16u) == 0));
            u64 reposj;
            if (narrow) {
                const u32 v32 = (u32)rv, inc = warp_incl_add(v32);
                const u32 lr = hr & (lt | (1u << lane));
                const u32 before = __shfl_sync(kFullMask, inc - v32, lr ? 31 - __clz(lr) : 0);
                reposj = lr ? (u64)(inc - before) : rcar + (u64)inc;
            } else {
                reposj = warp_seg_incl<u64>(hr, rv, rcar);
            }
            rcar = __shfl_sync(kFullMask, reposj, 31);
            if (valid) {
                if (sq & 8u) atomicOr(a.err, kErrBadStream);  // quad patches never occur
                u32 gx, gy, gz;
                if (!a.rp.hilbert) {
                    gx = gather3(reposj);
                    gy = gather3(reposj >> 1);
                    gz = gather3(reposj >> 2);
                } else if (reposj < (1ull << 18)) {
                    hilbert_xyz6(htab, (u32)reposj, a.rp.hstart_inv, gx, gy, gz);
                } else {
                    hilbert_xyz(htab, reposj, 20, 0u, gx, gy, gz);
                }
                cx = (i32)(pbx + ((quadj & 1u) >> 0) * 64u + gx);
                cy = (i32)(pby + ((quadj & 2u) >> 1) * 64u + gy);
                cz = (i32)(pbz + ((quadj & 4u) >> 2) * 64u + gz);
            }
        }
        // -rle: output position from the count prefix; -normal and cells: one per unit.
        u64 c = 1, opos = base + e;
        if (rle) {
            c = !valid ? 0ull : kept ? (u64)scnt[e] : (u64)max(a.counts[base + e], 0);
            const u64 incl = narrow ? (u64)warp_incl_add((u32)c) : warp_incl_add(c);
            opos = oc + incl - c;
            oc += __shfl_sync(kFullMask, incl, 31);
        }
        if (!valid) continue;  // after the round's warp-wide votes and shuffles
        if (a.rp.cells) {
            i32* co = reinterpret_cast<i32*>(a.out);
            co[3 * opos] = cx;
            co[3 * opos + 1] = cy;
            co[3 * opos + 2] = cz;
            continue;
        }
        float x, y, z;
        recover(q, cx, cy, cz, a.rp.off[0], a.rp.off[1], a.rp.off[2], x, y, z);
        if (opos + c > a.nout) {
            atomicOr(a.err, kErrOverflow);
            continue;
        }
        for (u64 k = 0; k < c; ++k) {
            a.out[3 * (opos + k)] = x;
            a.out[3 * (opos + k) + 1] = y;
            a.out[3 * (opos + k) + 2] = z;
        }
    }
}

inline int grid_cap(u64 n) {
    u64 b = (n + kThreads - 1) / kThreads;
    if (b < 1) b = 1;
    return (int)(b < 148ull * 8 ? b : 148ull * 8);
}

}  // namespace

void launch_block_streams(const uint32_t* words_blk, uint64_t base_blk, int width_blk, const uint32_t* words_cnt,
                          uint64_t base_cnt, int width_cnt, uint64_t nblocks, uint64_t units,
                          unsigned long long* blk_ids, uint8_t* is_start, uint32_t* start_block, LookBackState lb,
                          uint32_t* tile_counter, unsigned long long* count_total, uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((nblocks + kTile - 1) / kTile);
    if (!tiles) return;
    block_streams_kernel<<<tiles, kThreads, 0, st>>>(words_blk, base_blk, width_blk, words_cnt, base_cnt, width_cnt,
                                                     nblocks, units, blk_ids, is_start, start_block, lb, tile_counter,
                                                     count_total, err);
}

void launch_fill_u32(uint32_t* p, uint64_t n, uint32_t v, cudaStream_t st) {
    if (n) fill_u32_kernel<<<grid_cap(n), kThreads, 0, st>>>(p, n, v);
}
void launch_fill_u8(uint8_t* p, uint64_t n, uint8_t v, cudaStream_t st) {
    if (n) fill_u8_kernel<<<grid_cap(n), kThreads, 0, st>>>(p, n, v);
}
void launch_count_total(const int32_t* counts, uint64_t n, unsigned long long* total, cudaStream_t st) {
    if (n) count_total_kernel<<<grid_cap(n), kThreads, 0, st>>>(counts, n, total);
}
void launch_recover_units(const RecoverInputs& in, uint64_t units, uint64_t nout, RecoverParams rp,
                          const uint8_t* hilbert_inv_tab, uint32_t* flag, unsigned long long* agg,
                          unsigned long long* inc, uint32_t* tile_counter, float* out, uint32_t* err,
                          cudaStream_t st) {
    RecoverArgs a;
    a.rep_sym = in.rep_sym;
    a.rep_patch = in.rep_patch;
    a.npatch = in.npatch;
    a.quad_sym = in.quad_sym;
    a.is_start = in.is_start;
    a.start_block = in.start_block;
    a.blk_ids = in.blk_ids;
    a.nblocks = in.nblocks;
    a.counts = in.counts;
    a.rep_val = in.rep_val;
    a.units = units;
    a.nout = nout;
    a.rp = rp;
    a.hinv = hilbert_inv_tab;
    a.flag = flag;
    a.agg = agg;
    a.inc = inc;
    a.tile_counter = tile_counter;
    a.out = out;
    a.err = err;
    const unsigned tiles = (unsigned)((units + kTile - 1) / kTile);
    if (!tiles) return;
    if (rp.direct)
        recover_units_kernel<true><<<tiles, kThreads, 0, st>>>(a);
    else
        recover_units_kernel<false><<<tiles, kThreads, 0, st>>>(a);
}

}  // namespace dev
}  // namespace xnyz
