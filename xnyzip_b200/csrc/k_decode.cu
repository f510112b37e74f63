// Decompress-side kernels.
//
//   bitunpack      BitPacker<uint64_t>::unpack (encoder/bitpacking_encoder.hpp:53-80)
//   scan_u64       the prefix sums of block_decompressor.hpp:159-161 (u64, wrapping)
//   decode_stream  Huffman (huffman_encoder.hpp:205-243), Golomb-Rice (golomb_rice_encoder.hpp:
//                  150-192) and exp-Golomb (huffman_encoder.hpp:398-442) decoding of an
//                  unindexed bit stream in parallel, exact for any prefix code:
//                    1. each thread owns S bits and computes, for every entry offset e < L
//                       (L = longest codeword), where decoding from there leaves its S bits
//                       and how many codewords start inside (chains that meet an earlier
//                       chain's codeword boundary reuse its result);
//                    2. a block composes its 256 transition tables;
//                    3. blocks resolve their true entry offset by decoupled look-back over the
//                       predecessors' composed tables (function composition in registers);
//                    4. every thread decodes its S bits once from the true offset.
//                  An exit offset >= L (a codeword longer than L crossing a boundary) sets
//                  a flag and the host reruns the stream with decode_sequential.
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

// ------------------------------------------------------------------ bit unpack ----------
__global__ void __launch_bounds__(kThreads) bitunpack_kernel(const u32* __restrict__ words, u64 base, u64 n,
                                                             int width, u64* __restrict__ vals) {
    const u64 stride = (u64)gridDim.x * kThreads;
    const u64 mask = width >= 64 ? ~0ull : ((1ull << width) - 1);
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride)
        vals[i] = width ? (peek_lsb64(words, base + i * (u64)width) & mask) : 0ull;
}

// ------------------------------------------------------------------ scan ----------------
__global__ void __launch_bounds__(kThreads) scan_u64_kernel(const u64* __restrict__ in, u64* __restrict__ out, u64 n,
                                                            int exclusive, LookBackState lb, u32* tile_counter,
                                                            unsigned long long* total, u32* err) {
    __shared__ u64 sv[kTile];
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase;
    const u32 tile = claim_tile(tile_counter, &slot);
    const u64 base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, n - base);
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + threadIdx.x;
        if (e < cnt) sv[e] = in[base + e];
    }
    __syncthreads();
    const u32 e0 = threadIdx.x * kItems;
    u64 s = 0;
    for (int i = 0; i < kItems; ++i)
        if (e0 + i < cnt) s += sv[e0 + i];
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(s, 0ull, AddOp{}, scratch, tot);
    if (threadIdx.x == 0) {
        LookBack64 l{lb.flag, lb.agg, lb.inc};
        const u64 before = lookback_add(l, tile, tot, err);
        sbase = before;
        if (tile == gridDim.x - 1 && total) *total = before + tot;
    }
    __syncthreads();
    u64 run = sbase + ex;
    for (int i = 0; i < kItems; ++i)
        if (e0 + i < cnt) {
            const u64 v = sv[e0 + i];
            sv[e0 + i] = exclusive ? run : run + v;
            run += v;
        }
    __syncthreads();
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + threadIdx.x;
        if (e < cnt) out[base + e] = sv[e];
    }
}

// ---------------------------------------------------------------- codewords -------------
// A stream starts `base` bits into `words` (containers place streams at byte offsets).
struct Stream {
    const u32* words;
    u64 base;
    u64 total_bits;
    DecodeTable t;
};

// Huffman: primary table lookup, tree walk for codes longer than root_bits.  Returns the
// length (0 marks an invalid code) and the symbol.
__device__ __forceinline__ u32 huff_one(const Stream& s, u64 p, u32& sym) {
    const u32 w = peek_msb32(s.words, s.base + p);
    const u32 e = __ldg(&s.t.root[w >> (32 - s.t.root_bits)]);
    if (!(e & 0x80000000u)) {
        sym = e & 0xffffffu;
        return e >> 24;
    }
    u32 node = e & 0x7fffffffu;
    for (u32 i = (u32)s.t.root_bits; i < 32u; ++i) {
        const u32 c = __ldg(&s.t.tree[2 * node + ((w >> (31u - i)) & 1u)]);
        if (c & 0x80000000u) {
            sym = c & 0x7fffffffu;
            return c == 0xffffffffu ? 0u : i + 1;
        }
        node = c;
    }
    sym = 0;
    return 0;
}

// Golomb-Rice (LSB-first): q ones, a zero, k remainder bits.
__device__ __forceinline__ u64 gr_one(const Stream& s, u64 p, u64& val) {
    const int k = s.t.param;
    u64 q = 0;
    u64 v = peek_lsb64(s.words, s.base + p);
    while (v == ~0ull) {
        q += 64;
        if (p + q >= s.total_bits + 64) {  // a run past the end of the stream: invalid
            val = 0;
            return s.total_bits + 1 - p;
        }
        v = peek_lsb64(s.words, s.base + p + q);
    }
    q += (u64)(__ffsll((long long)~v) - 1);
    if (p + q + 1 + (u64)k > s.total_bits) {  // codeword would end past the stream: invalid
        val = 0;
        return s.total_bits + 1 - p;
    }
    const u64 r = k ? (peek_lsb64(s.words, s.base + p + q + 1) & ((1ull << k) - 1)) : 0ull;
    val = (q << k) + r;
    return q + 1 + (u64)k;
}

// exp-Golomb (MSB-first): z zeros, n1 in z+1 bits, then k bits least significant first.
__device__ __forceinline__ u64 eg_one(const Stream& s, u64 p, u64& val) {
    const int k = s.t.param;
    u64 z = 0;
    const u64 q0 = s.base + p;
    u32 w = peek_msb32(s.words, q0);
    while (w == 0u) {
        z += 32;
        if (p + z >= s.total_bits + 64) {  // a zero run past the end of the stream: invalid
            val = 0;
            return s.total_bits + 1 - p;
        }
        w = peek_msb32(s.words, q0 + z);
    }
    z += (u64)__clz((int)w);
    if (p + 2 * z + 1 + (u64)k > s.total_bits) {  // codeword would end past the stream: invalid
        val = 0;
        return s.total_bits + 1 - p;
    }
    u64 n1;
    if (z + 1 <= 32) {
        n1 = peek_msb32(s.words, q0 + z) >> (31 - z);
    } else {
        const u64 hi = peek_msb32(s.words, q0 + z);
        const u64 lo = peek_msb32(s.words, q0 + z + 32);
        n1 = z + 1 >= 64 ? ~0ull : (((hi << 32) | lo) >> (63 - z));
    }
    const u64 rb = k ? (peek_msb32(s.words, q0 + 2 * z + 1) >> (32 - k)) : 0ull;
    const u64 low = k ? (u64)(__brev((u32)rb) >> (32 - k)) : 0ull;
    const u64 u = ((n1 - 1) << k) | low;
    // from_unsigned of signed symbol types: zigzag decode (huffman_encoder.hpp:315-333)
    val = s.t.zigzag ? ((u >> 1) ^ (~(u & 1ull) + 1ull)) : u;
    return 2 * z + 1 + (u64)k;
}

template <int KIND>
__device__ __forceinline__ u64 codeword(const Stream& s, u64 p, u64& val) {
    if (KIND == kCodeHuffman) {
        u32 sym;
        const u32 l = huff_one(s, p, sym);
        val = l ? __ldg(&s.t.symvals[sym]) : 0ull;
        return l ? l : (u64)(1u << 20);  // invalid code: jump far so the chain ends; flagged on write
    } else if (KIND == kCodeGolombRice) {
        return gr_one(s, p, val);
    } else {
        return eg_one(s, p, val);
    }
}

// ------------------------------------------------------------- stream decoder -----------
constexpr int kMaxL = 64;
constexpr u32 kOOD = 0xffu;
constexpr int kSubBits = 2048;  // bits per subsequence (one thread)
constexpr int kWinBits = 512;   // chains are merged within the first kWinBits of a subsequence
constexpr int kBmWords = kWinBits / 32;
static_assert(kSubBits == kDecodeSubBits && kThreads == kDecodeBlockSubs && kMaxL == kDecodeMaxL, "decode geometry");

struct DecodeShared {
    u8 fx[kMaxL * kThreads];     // [e][t]: exit offset into the next subsequence or kOOD
    u16 fc[kMaxL * kThreads];    // [e][t]: codewords starting inside
    u32 bm[2 * kBmWords * kThreads];  // [root][word][t]: codeword starts of two root chains
    u64 sstart[kThreads];   // true entry offset of each subsequence (any value)
    u64 scount[kThreads];   // codewords before it
    u32 slot;
};

__device__ __forceinline__ bool bm_test(const u32* bm, int r, u32 q) {
    return (bm[(r * kBmWords + (q >> 5)) * kThreads + threadIdx.x] >> (q & 31u)) & 1u;
}
__device__ __forceinline__ void bm_set(u32* bm, int r, u32 q) {
    bm[(r * kBmWords + (q >> 5)) * kThreads + threadIdx.x] |= 1u << (q & 31u);
}
__device__ __forceinline__ u32 bm_popc_below(const u32* bm, int r, u32 q) {
    u32 c = 0;
    for (u32 w = 0; w < (q >> 5); ++w) c += __popc(bm[(r * kBmWords + w) * kThreads + threadIdx.x]);
    const u32 rem = q & 31u;
    if (rem) c += __popc(bm[(r * kBmWords + (q >> 5)) * kThreads + threadIdx.x] & ((1u << rem) - 1u));
    return c;
}

struct DecodeArgs {
    Stream s;
    u64 nsub;
    int L;               // entry offsets tracked, or
    const u32* L_run;    // if set: L = min(64, longest one-run + 1 + k)  (Golomb-Rice)
    u64 nsym;
    int out_width;
    void* out;
    u32* flag;
    u64* agg;   // [tile][kMaxL]: exit | count << 8
    u64* inc;   // [tile][2]: exit, count through the tile
    u32* tile_counter;
    u32* err;
    u32* need_fallback;
    unsigned long long* total_codewords;
};

__device__ __forceinline__ void store_sym(void* out, int width, u64 i, u64 v) {
    if (width == 1) static_cast<u8*>(out)[i] = (u8)v;
    else if (width == 4) static_cast<u32*>(out)[i] = (u32)v;
    else static_cast<u64*>(out)[i] = v;
}

// One-bits of an LSB-first stream from stream position p up to the first zero.
__device__ __forceinline__ u64 lead_ones(const Stream& s, u64 p) {
    u64 q = 0;
    while (p + q < s.total_bits) {
        const u64 v = peek_lsb64(s.words, s.base + p + q);
        if (v != ~0ull) return q + (u64)(__ffsll((long long)~v) - 1);
        q += 64;
    }
    return q;
}

// Entry offsets tracked per subsequence.  Golomb-Rice: a codeword crossing into subsequence s
// ends at an offset x <= k, or its terminating zero lies inside s after a run of ones that
// reaches back to s's first bit, so x = k + 1 + (leading ones of s): k + 2 entries, the last
// one "special".  Other codes: offsets 0 .. L-1.
template <int KIND>
__device__ __forceinline__ u32 entry_index(u64 x, int L, int k) {
    if (KIND == kCodeGolombRice) return x <= (u64)k ? (u32)x : (u32)(k + 1);
    return x < (u64)L ? (u32)x : kOOD;
}
template <int KIND>
__device__ __forceinline__ u64 entry_offset(const Stream& s, u32 i, u64 Bsub, int k) {
    if (KIND == kCodeGolombRice && i == (u32)(k + 1)) return (u64)k + 1 + lead_ones(s, Bsub);
    return i;
}

template <int KIND>
__global__ void __launch_bounds__(kThreads) decode_stream_kernel(DecodeArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    DecodeShared& sh = *reinterpret_cast<DecodeShared*>(smem_raw);
    const u32 tile = claim_tile(a.tile_counter, &sh.slot);
    const int t = threadIdx.x;
    const u64 s = (u64)tile * kThreads + t;
    const u64 first_sub = (u64)tile * kThreads;
    const u32 nvalid = (u32)min((u64)kThreads, a.nsub - first_sub);
    const int gk = a.s.t.param;
    const int L = KIND == kCodeGolombRice ? min(kMaxL, gk + 2) : a.L;
    const u64 B = s * kSubBits;
    const u64 Bend = min(B + kSubBits, a.s.total_bits);

    // ---- 1. transition table of my subsequence ----
    if ((u32)t < nvalid) {
        u32 rx[2] = {0, 0}, rc[2] = {0, 0};
        int nroots = 0;
        for (int e = 0; e < L; ++e) {
            const u64 off = entry_offset<KIND>(a.s, (u32)e, B, gk);
            u64 p = B + off;
            u32 ox = kOOD, oc = 0;
            if (p >= Bend) {  // no codeword starts here: the entry passes through
                ox = Bend == B + kSubBits ? entry_index<KIND>(off - kSubBits, L, gk) : kOOD;
                sh.fx[e * kThreads + t] = (u8)ox;
                sh.fc[e * kThreads + t] = 0;
                continue;
            }
            int hit = -1;
            if (off < (u64)kWinBits)
                for (int r = 0; r < nroots; ++r)
                    if (bm_test(sh.bm, r, (u32)off)) hit = r;
            if (hit >= 0) {
                ox = rx[hit];
                oc = rc[hit] - bm_popc_below(sh.bm, hit, (u32)off);
            } else {
                const bool rec = nroots < 2 && off < (u64)kWinBits;
                if (rec) {
                    for (int w = 0; w < kBmWords; ++w) sh.bm[(nroots * kBmWords + w) * kThreads + t] = 0;
                    bm_set(sh.bm, nroots, (u32)off);
                }
                u32 c = 0;
                bool merged = false;
                while (p < Bend) {
                    u64 v;
                    p += codeword<KIND>(a.s, p, v);
                    ++c;
                    if (p < Bend && p - B < (u64)kWinBits) {
                        const u32 q = (u32)(p - B);
                        for (int r = 0; r < nroots && !merged; ++r)
                            if (bm_test(sh.bm, r, q)) {
                                merged = true;
                                ox = rx[r];
                                oc = c + rc[r] - bm_popc_below(sh.bm, r, q);
                            }
                        if (merged) break;
                        if (rec) bm_set(sh.bm, nroots, q);
                    }
                }
                if (!merged) {
                    ox = (Bend == B + kSubBits && p >= Bend) ? entry_index<KIND>(p - (B + kSubBits), L, gk) : kOOD;
                    oc = c;
                    if (rec) {
                        rx[nroots] = ox;
                        rc[nroots] = c;
                        ++nroots;
                    }
                }
            }
            sh.fx[e * kThreads + t] = (u8)ox;
            sh.fc[e * kThreads + t] = (u16)oc;
        }
    }
    __syncthreads();

    // ---- 2. composed table of the block (warp 0; lane holds entries lane and lane+32) ----
    // ---- 3. look-back over predecessor blocks ----
    // ---- 4. true entry of every subsequence (lane 0 walks the tables; entries outside a
    //         table, i.e. after a codeword longer than L crossed the boundary, are decoded
    //         on the spot, so the result is exact for any code) ----
    if (t < 32) {
        u32 gx[2];
        u64 gc[2];
        for (int h = 0; h < 2; ++h) {
            const int e = t + 32 * h;
            u32 x = e < L ? (u32)e : kOOD;
            u64 c = 0;
            for (u32 j = 0; j < nvalid && x != kOOD; ++j) {
                c += sh.fc[x * kThreads + j];
                x = sh.fx[x * kThreads + j];
            }
            gx[h] = x;
            gc[h] = c;
        }
        u64 E = 0, C = 0;
        bool failed = false;
        if (tile > 0) {
            for (int h = 0; h < 2; ++h) {
                const int e = t + 32 * h;
                st_volatile(&a.agg[(u64)tile * kMaxL + e], (u64)gx[h] | (gc[h] << 8));
            }
            __threadfence();
            __syncwarp();
            if (t == 0) st_volatile(&a.flag[tile], 1u);
            // G: composition of the aggregates walked so far (identity to start).
            u32 Gx[2] = {(u32)t, (u32)t + 32};
            u64 Gc[2] = {0, 0};
            long long p = (long long)tile - 1;
            u32 spins = 0;
            bool need_pred = false;
            while (true) {
                u32 f = 0;
                if (t == 0) f = ld_volatile(&a.flag[p]);
                f = __shfl_sync(kFullMask, f, 0);
                if (f == 0) {
                    if (++spins > kSpinLimit) {
                        failed = true;
                        break;
                    }
                    if (spins > 64) __nanosleep(100);
                    continue;
                }
                __threadfence();
                if (f == 2) {
                    const u64 X = ld_volatile(&a.inc[(u64)p * 2]);
                    const u64 CX = ld_volatile(&a.inc[(u64)p * 2 + 1]);
                    if (p == (long long)tile - 1) {  // exact entry from the direct predecessor
                        E = X;
                        C = CX;
                        break;
                    }
                    const u32 Xi = entry_index<KIND>(X, L, gk);
                    const u32 Xs = Xi == kOOD ? 0u : Xi;
                    const u32 ex0 = __shfl_sync(kFullMask, Gx[0], Xs & 31u), ex1 = __shfl_sync(kFullMask, Gx[1], Xs & 31u);
                    const u64 ec0 = __shfl_sync(kFullMask, Gc[0], Xs & 31u), ec1 = __shfl_sync(kFullMask, Gc[1], Xs & 31u);
                    const u32 gxX = Xs < 32u ? ex0 : ex1;
                    if (Xi == kOOD || gxX == kOOD) {
                        need_pred = true;  // the composition does not cover this entry
                    } else {
                        E = gxX;
                        C = CX + (Xs < 32u ? ec0 : ec1);
                    }
                    break;
                }
                // Aggregate F of block p: G <- G o F (both halves read G before either is
                // overwritten).
                {
                    u32 nx[2];
                    u64 nc[2];
                    for (int h = 0; h < 2; ++h) {
                        const u64 fv = ld_volatile(&a.agg[(u64)p * kMaxL + t + 32 * h]);
                        const u32 y = (u32)(fv & 0xffu);
                        const u32 yy = y == kOOD ? 0u : y;
                        const u32 gx0 = __shfl_sync(kFullMask, Gx[0], yy & 31u), gx1 = __shfl_sync(kFullMask, Gx[1], yy & 31u);
                        const u64 gc0 = __shfl_sync(kFullMask, Gc[0], yy & 31u), gc1 = __shfl_sync(kFullMask, Gc[1], yy & 31u);
                        nx[h] = y == kOOD ? kOOD : (yy < 32u ? gx0 : gx1);
                        nc[h] = (fv >> 8) + (yy < 32u ? gc0 : gc1);
                    }
                    for (int h = 0; h < 2; ++h) {
                        Gx[h] = (t + 32 * h < L) ? nx[h] : kOOD;
                        Gc[h] = nc[h];
                    }
                }
                --p;
                if (p < 0) {  // cannot happen: tile 0 always publishes its inclusive value
                    failed = true;
                    break;
                }
            }
            if (need_pred && !failed) {
                // Wait for the direct predecessor's exact exit.
                spins = 0;
                while (true) {
                    u32 f = 0;
                    if (t == 0) f = ld_volatile(&a.flag[tile - 1]);
                    f = __shfl_sync(kFullMask, f, 0);
                    if (f == 2u) break;
                    if (++spins > kSpinLimit) {
                        failed = true;
                        break;
                    }
                    if (spins > 64) __nanosleep(100);
                }
                __threadfence();
                if (!failed) {
                    E = ld_volatile(&a.inc[(u64)(tile - 1) * 2]);
                    C = ld_volatile(&a.inc[(u64)(tile - 1) * 2 + 1]);
                }
            }
        }
        // Fast path: my composed table covers E -> publish my inclusive value right away.
        // (E is an entry index when it came from a composed table, an offset when it came from
        // a predecessor's walk; entry_index maps both.)
        const u32 Ei = entry_index<KIND>(E, L, gk);
        const u32 Es = Ei == kOOD ? 0u : Ei;
        const u32 mx0 = __shfl_sync(kFullMask, gx[0], Es & 31u), mx1 = __shfl_sync(kFullMask, gx[1], Es & 31u);
        const u64 mc0 = __shfl_sync(kFullMask, gc[0], Es & 31u), mc1 = __shfl_sync(kFullMask, gc[1], Es & 31u);
        const u32 tabX = Es < 32u ? mx0 : mx1;
        const bool fast = !failed && Ei != kOOD && tabX != kOOD;
        if (t == 0) {
            if (failed) {
                atomicOr(a.err, kErrTimeout);
                atomicOr(a.need_fallback, 1u);
            }
            if (fast) {
                st_volatile(&a.inc[(u64)tile * 2], (u64)tabX);
                st_volatile(&a.inc[(u64)tile * 2 + 1], C + (Es < 32u ? mc0 : mc1));
                __threadfence();
                st_volatile(&a.flag[tile], 2u);
            }
            // walk my subsequences from the true entry (x: offset into subsequence j)
            u64 x = E;
            if (KIND == kCodeGolombRice && E > (u64)gk) x = entry_offset<KIND>(a.s, (u32)(gk + 1), first_sub * kSubBits, gk);
            u64 c = C;
            for (u32 j = 0; j < nvalid; ++j) {
                sh.sstart[j] = x;
                sh.scount[j] = c;
                const u32 xi = entry_index<KIND>(x, L, gk);
                if (xi != kOOD && sh.fx[xi * kThreads + j] != kOOD) {
                    c += sh.fc[xi * kThreads + j];
                    const u32 ni = sh.fx[xi * kThreads + j];
                    x = entry_offset<KIND>(a.s, ni, (first_sub + j + 1) * kSubBits, gk);
                } else {
                    const u64 Bj = (first_sub + j) * kSubBits;
                    const u64 Ej = min(Bj + kSubBits, a.s.total_bits);
                    u64 pp = Bj + x;
                    while (pp < Ej) {
                        u64 v;
                        pp += codeword<KIND>(a.s, pp, v);
                        ++c;
                    }
                    x = pp >= Bj + kSubBits ? pp - (Bj + kSubBits) : 0ull;
                }
            }
            if (!fast) {
                st_volatile(&a.inc[(u64)tile * 2], x);
                st_volatile(&a.inc[(u64)tile * 2 + 1], c);
                __threadfence();
                st_volatile(&a.flag[tile], 2u);
            }
            if (tile == gridDim.x - 1) *a.total_codewords = c;
        }
    }
    __syncthreads();

    // ---- 5. decode my subsequence from its true entry ----
    if ((u32)t < nvalid) {
        u64 idx = sh.scount[t];
        u64 p = B + sh.sstart[t];
        while (p < Bend && idx < a.nsym) {
            u64 v;
            const u64 len = codeword<KIND>(a.s, p, v);
            if (p + len > a.s.total_bits || (KIND == kCodeHuffman && len >= (1u << 20))) {
                atomicOr(a.err, kErrBadStream);
                return;
            }
            store_sym(a.out, a.out_width, idx, v);
            ++idx;
            p += len;
        }
    }
}

template <int KIND>
__global__ void decode_sequential_kernel(Stream s, u64 nsym, int width, void* out, unsigned long long* total, u32* err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    u64 p = 0, i = 0;
    while (i < nsym && p < s.total_bits) {
        u64 v;
        const u64 len = codeword<KIND>(s, p, v);
        if (p + len > s.total_bits || (KIND == kCodeHuffman && len >= (1u << 20))) {
            atomicOr(err, kErrBadStream);
            break;
        }
        store_sym(out, width, i, v);
        ++i;
        p += len;
    }
    *total = i;
}

// ---------------------------------------------------------------- units --------------
__global__ void __launch_bounds__(kThreads) block_starts_kernel(const u64* __restrict__ start_excl,
                                                                const u64* __restrict__ blk_cnt_unused, u64 nb,
                                                                u64 units, u8* __restrict__ is_start,
                                                                u32* __restrict__ start_block, u32* err) {
    (void)blk_cnt_unused;
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 b = (u64)blockIdx.x * kThreads + threadIdx.x; b < nb; b += stride) {
        const u64 st = start_excl[b];
        const u64 en = (b + 1 < nb) ? start_excl[b + 1] : units;
        if (en > st && st < units) {  // non-empty block; empty ones are skipped like the reference
            is_start[st] = 1;
            start_block[st] = (u32)b;
        }
    }
}


// ---------------------------------------------------------------- helpers --------------
__global__ void fill_u64_kernel(u64* p, u64 n, u64 v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void fill_u32_kernel(u32* p, u64 n, u32 v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}
__global__ void fill_u8_kernel(u8* p, u64 n, u8 v) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) p[i] = v;
}

// Longest run of one-bits in an LSB-first stream (bounds the Golomb-Rice codeword length).
// Each thread scans 64 words and follows a run that crosses its chunk end for up to 8 more
// words; longer runs only need to be recognised as longer than 64 bits.
__global__ void max_ones_run_kernel(const u32* __restrict__ words, u64 nwords, u32* out) {
    const u64 chunk = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 w0 = chunk * 64;
    if (w0 >= nwords) return;
    const u64 w1 = min(nwords, w0 + 64), w2 = min(nwords, w1 + 8);
    u32 run = 0, best = 0;
    for (u64 w = w0; w < w2; ++w) {
        const u32 x = words[w];
        if (x == 0xffffffffu) {
            run += 32;
            continue;
        }
        run += (u32)(__ffs((int)~x) - 1);
        best = max(best, run);
        if (w >= w1) {
            run = 0;
            break;
        }
        u32 y = x, r = 0;
        while (y) {
            y &= y >> 1;
            ++r;
        }
        best = max(best, r);
        run = (u32)__clz((int)~x);
    }
    best = max(best, run);
    atomicMax(out, best);
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
__device__ __forceinline__ Seg shfl_up_seg(Seg v, int d) {
    return Seg{__shfl_up_sync(kFullMask, v.head, d), __shfl_up_sync(kFullMask, v.sum, d)};
}

// Block-wide exclusive scan of Seg values.
__device__ Seg block_exclusive_seg(Seg v, Seg* scratch, Seg& total) {
    SegOp op;
    const int w = threadIdx.x >> 5;
    Seg inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Seg o = shfl_up_seg(inc, d);
        if ((int)lane_id() >= d) inc = op(o, inc);
    }
    if (lane_id() == 31) scratch[w] = inc;
    __syncthreads();
    if (w == 0) {
        Seg x = (int)lane_id() < kThreads / 32 ? scratch[lane_id()] : Seg{0, 0};
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const Seg o = shfl_up_seg(x, d);
            if ((int)lane_id() >= d) x = op(o, x);
        }
        if ((int)lane_id() < kThreads / 32) scratch[lane_id()] = x;
    }
    __syncthreads();
    const Seg wp = w == 0 ? Seg{0, 0} : scratch[w - 1];
    Seg ex = shfl_up_seg(inc, 1);
    if (lane_id() == 0) ex = Seg{0, 0};
    total = scratch[kThreads / 32 - 1];
    const Seg r = op(wp, ex);
    __syncthreads();
    return r;
}

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

template <bool DIRECT>
__global__ void __launch_bounds__(kThreads) recover_units_kernel(RecoverArgs a) {
    __shared__ u8 srep[kTile];
    __shared__ u8 squad[DIRECT ? 1 : kTile];
    __shared__ u8 sstart[DIRECT ? 1 : kTile];
    __shared__ u64 scr64[16];
    __shared__ Seg scrseg[16];
    __shared__ u32 slot;
    __shared__ u64 base_zero, base_count, base_sfc;
    __shared__ Seg base_quad, base_blk, base_rep;
    __shared__ u8 htab[256];

    const u32 tile = claim_tile(a.tile_counter, &slot);
    const u32 ntiles = gridDim.x;
    const u64 base = (u64)tile * kTile;
    const u32 cnt = (u32)min((u64)kTile, a.units - base);
    const int tid = threadIdx.x;
    for (int i = tid; i < 256; i += kThreads) htab[i] = a.hinv ? a.hinv[i] : 0;
    for (int i = 0; i < kItems; ++i) {
        const u32 e = (u32)i * kThreads + tid;
        if (e < cnt) {
            srep[e] = a.rep_sym[base + e];
            if (!DIRECT) {
                squad[e] = a.quad_sym[base + e];
                sstart[e] = a.is_start[base + e];
            }
        }
    }
    __syncthreads();
    const u32 e0 = (u32)tid * kItems;
    const bool rle = a.rp.rle != 0;

    // ---- round 1: zero symbols, quad segments, block carry, counts ----
    u64 zr = 0, csum = 0;
    Seg qs{0, 0}, bs{0, 0};
    SegOp op;
    for (int i = 0; i < kItems; ++i) {
        const u32 e = e0 + i;
        if (e >= cnt) break;
        zr += srep[e] == 0;
        if (rle) csum += (u64)max(a.counts[base + e], 0);
        if (!DIRECT) {
            const bool st = sstart[e] != 0;
            qs = op(qs, Seg{st ? 1ull : 0ull, (u64)(squad[e] ? squad[e] - 1u : 0u)});
            bs = op(bs, Seg{st ? 1ull : 0ull, st ? (u64)a.start_block[base + e] : 0ull});
        }
    }
    u64 tz, tc;
    const u64 ez = block_exclusive<kThreads>(zr, 0ull, AddOp{}, scr64, tz);
    const u64 ec = block_exclusive<kThreads>(csum, 0ull, AddOp{}, scr64, tc);
    Seg tq{0, 0}, tb{0, 0}, eq{0, 0}, eb{0, 0};
    if (!DIRECT) {
        eq = block_exclusive_seg(qs, scrseg, tq);
        eb = block_exclusive_seg(bs, scrseg, tb);
    }
    if (tid == 0) {
        LookBack64 l{a.flag, a.agg, a.inc};
        base_zero = lookback_add(l, tile, tz, a.err);
    } else if (tid == 32 && rle) {
        LookBack64 l{a.flag + ntiles, a.agg + 2ull * ntiles, a.inc + 2ull * ntiles};
        base_count = lookback_add(l, tile, tc, a.err);
    } else if (tid == 64 && !DIRECT) {
        Seg* ag = reinterpret_cast<Seg*>(a.agg + 4ull * ntiles);
        Seg* in = reinterpret_cast<Seg*>(a.inc + 4ull * ntiles);
        base_quad = lookback(a.flag + 2 * ntiles, ag, in, tile, tq, Seg{0, 0}, SegOp{}, LoadSeg{}, StoreSeg{}, a.err);
    } else if (tid == 96 && !DIRECT) {
        Seg* ag = reinterpret_cast<Seg*>(a.agg + 6ull * ntiles);
        Seg* in = reinterpret_cast<Seg*>(a.inc + 6ull * ntiles);
        base_blk = lookback(a.flag + 3 * ntiles, ag, in, tile, tb, Seg{0, 0}, SegOp{}, LoadSeg{}, StoreSeg{}, a.err);
    }
    if (!rle && tid == 0) base_count = 0;
    __syncthreads();

    // ---- round 2: repos values (need the patch index) -> repos segments / SFC sums ----
    u64 zrun = base_zero + ez;
    u64 rv[kItems];
    Seg rs{0, 0};
    u64 dsum = 0;
    for (int i = 0; i < kItems; ++i) {
        const u32 e = e0 + i;
        rv[i] = 0;
        if (e >= cnt) continue;
        const u32 sym = srep[e];
        u64 v;
        if (sym == 0) {
            if (zrun < a.npatch) {
                v = a.rep_patch[zrun];
            } else {
                v = 0;
                atomicOr(a.err, kErrBadStream);
            }
            ++zrun;
        } else {
            v = sym - 1u;
        }
        rv[i] = v;
        if (DIRECT) {
            dsum += v;
        } else {
            const bool st = sstart[e] != 0;
            const bool qchange = squad[e] != 1;  // quad delta != 0
            rs = op(rs, Seg{(st || qchange) ? 1ull : 0ull, v});
        }
    }
    u64 td = 0, ed = 0;
    Seg tr{0, 0}, er{0, 0};
    if (DIRECT) ed = block_exclusive<kThreads>(dsum, 0ull, AddOp{}, scr64, td);
    else er = block_exclusive_seg(rs, scrseg, tr);
    if (tid == 0) {
        if (DIRECT) {
            LookBack64 l{a.flag + 4 * ntiles, a.agg + 8ull * ntiles, a.inc + 8ull * ntiles};
            base_sfc = lookback_add(l, tile, td, a.err);
        } else {
            Seg* ag = reinterpret_cast<Seg*>(a.agg + 8ull * ntiles);
            Seg* in = reinterpret_cast<Seg*>(a.inc + 8ull * ntiles);
            base_rep = lookback(a.flag + 4 * ntiles, ag, in, tile, tr, Seg{0, 0}, SegOp{}, LoadSeg{}, StoreSeg{}, a.err);
        }
    }
    __syncthreads();

    // ---- final: coordinates, recover, unshift, expand ----
    const QuantParams q = a.rp.q;
    // -rle: output position from the count prefix; -normal: one point per unit.
    u64 opos = rle ? base_count + ec : base + e0;
    u64 sfc = base_sfc + ed;
    Seg qrun = op(base_quad, eq), brun = op(base_blk, eb), rrun = op(base_rep, er);
    for (int i = 0; i < kItems; ++i) {
        const u32 e = e0 + i;
        if (e >= cnt) break;
        i32 cx, cy, cz;
        if (DIRECT) {
            sfc += rv[i];
            const u64 m = a.rp.hilbert ? hilbert_apply(htab, sfc, a.rp.bits, 0u) : sfc;
            cx = (i32)gather3(m);
            cy = (i32)gather3(m >> 1);
            cz = (i32)gather3(m >> 2);
        } else {
            const bool st = sstart[e] != 0;
            qrun = op(qrun, Seg{st ? 1ull : 0ull, (u64)(squad[e] ? squad[e] - 1u : 0u)});
            brun = op(brun, Seg{st ? 1ull : 0ull, st ? (u64)a.start_block[base + e] : 0ull});
            rrun = op(rrun, Seg{(st || squad[e] != 1) ? 1ull : 0ull, rv[i]});
            const u64 quadj = qrun.sum, reposj = rrun.sum, b = brun.sum;
            if (squad[e] == 0) atomicOr(a.err, kErrBadStream);  // quad patches never occur
            const u64 blk = b < a.nblocks ? a.blk_ids[b] : 0ull;
            const u64 nx = a.rp.nx, ny = a.rp.ny;
            const u64 pbx = (blk % nx * 2) * 64, pby = (blk / nx % ny * 2) * 64, pbz = (blk / nx / ny * 2) * 64;
            u64 m = reposj;
            if (a.rp.hilbert)
                m = reposj < (1ull << 18) ? hilbert_apply(htab, reposj, 5, a.rp.hstart_inv)
                                          : hilbert_apply(htab, reposj, 20, 0u);
            cx = (i32)(pbx + ((quadj & 1u) >> 0) * 64 + (u64)gather3(m));
            cy = (i32)(pby + ((quadj & 2u) >> 1) * 64 + (u64)gather3(m >> 1));
            cz = (i32)(pbz + ((quadj & 4u) >> 2) * 64 + (u64)gather3(m >> 2));
        }
        float x, y, z;
        recover(q, cx, cy, cz, a.rp.off[0], a.rp.off[1], a.rp.off[2], x, y, z);
        const u64 c = rle ? (u64)max(a.counts[base + e], 0) : 1ull;
        if (opos + c > a.nout) {
            atomicOr(a.err, kErrOverflow);
            break;
        }
        for (u64 r = 0; r < c; ++r) {
            a.out[3 * (opos + r)] = x;
            a.out[3 * (opos + r) + 1] = y;
            a.out[3 * (opos + r) + 2] = z;
        }
        opos += c;
    }
}

inline int grid_cap(u64 n) {
    u64 b = (n + kThreads - 1) / kThreads;
    if (b < 1) b = 1;
    return (int)(b < 148ull * 8 ? b : 148ull * 8);
}

}  // namespace

void launch_bitunpack(const uint32_t* words, uint64_t base_bits, uint64_t n, int width, unsigned long long* vals,
                      cudaStream_t st) {
    u64 blocks = (n + kThreads - 1) / kThreads;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (!blocks) return;
    bitunpack_kernel<<<(unsigned)blocks, kThreads, 0, st>>>(words, base_bits, n, width, vals);
}

void launch_scan_u64(const unsigned long long* in, unsigned long long* out, uint64_t n, int exclusive,
                     LookBackState lb, uint32_t* tile_counter, unsigned long long* total, uint32_t* err,
                     cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kTile - 1) / kTile);
    if (!tiles) return;
    scan_u64_kernel<<<tiles, kThreads, 0, st>>>(in, out, n, exclusive, lb, tile_counter, total, err);
}


void launch_fill_u64(unsigned long long* p, uint64_t n, unsigned long long v, cudaStream_t st) {
    if (n) fill_u64_kernel<<<grid_cap(n), kThreads, 0, st>>>(p, n, v);
}
void launch_fill_u32(uint32_t* p, uint64_t n, uint32_t v, cudaStream_t st) {
    if (n) fill_u32_kernel<<<grid_cap(n), kThreads, 0, st>>>(p, n, v);
}
void launch_fill_u8(uint8_t* p, uint64_t n, uint8_t v, cudaStream_t st) {
    if (n) fill_u8_kernel<<<grid_cap(n), kThreads, 0, st>>>(p, n, v);
}
void launch_max_ones_run(const uint32_t* words, uint64_t nwords, uint32_t* out, cudaStream_t st) {
    const u64 chunks = (nwords + 63) / 64;
    if (chunks) max_ones_run_kernel<<<(unsigned)((chunks + 255) / 256), 256, 0, st>>>(words, nwords, out);
}
void launch_count_total(const int32_t* counts, uint64_t n, unsigned long long* total, cudaStream_t st) {
    if (n) count_total_kernel<<<grid_cap(n), kThreads, 0, st>>>(counts, n, total);
}
void launch_block_starts(const unsigned long long* start_excl, uint64_t nblocks, uint64_t units, uint8_t* is_start,
                         uint32_t* start_block, uint32_t* err, cudaStream_t st) {
    if (nblocks)
        block_starts_kernel<<<grid_cap(nblocks), kThreads, 0, st>>>(start_excl, nullptr, nblocks, units, is_start,
                                                                    start_block, err);
}

size_t decode_smem_bytes() { return sizeof(DecodeShared); }

void launch_decode_stream(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits, DecodeTable t,
                          int L, const uint32_t* L_run, uint64_t nsym, int out_width, void* out, uint32_t* flag,
                          unsigned long long* agg, unsigned long long* inc, uint32_t* tile_counter, uint32_t* err,
                          uint32_t* need_fallback, unsigned long long* total_codewords, cudaStream_t st) {
    DecodeArgs a;
    a.s = Stream{words, base_bits, total_bits, t};
    a.nsub = (total_bits + kSubBits - 1) / kSubBits;
    a.L = L < 1 ? 1 : (L > kMaxL ? kMaxL : L);
    a.L_run = L_run;
    a.nsym = nsym;
    a.out_width = out_width;
    a.out = out;
    a.flag = flag;
    a.agg = agg;
    a.inc = inc;
    a.tile_counter = tile_counter;
    a.err = err;
    a.need_fallback = need_fallback;
    a.total_codewords = total_codewords;
    const unsigned tiles = (unsigned)((a.nsub + kThreads - 1) / kThreads);
    if (!tiles) return;
    const int smem = (int)sizeof(DecodeShared);
    if (kind == kCodeHuffman) {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeHuffman>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_stream_kernel<kCodeHuffman><<<tiles, kThreads, smem, st>>>(a);
    } else if (kind == kCodeGolombRice) {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeGolombRice>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_stream_kernel<kCodeGolombRice><<<tiles, kThreads, smem, st>>>(a);
    } else {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeExpGolomb>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        decode_stream_kernel<kCodeExpGolomb><<<tiles, kThreads, smem, st>>>(a);
    }
}

void launch_decode_sequential(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits,
                              DecodeTable t, uint64_t nsym, int out_width, void* out,
                              unsigned long long* total_codewords, uint32_t* err, cudaStream_t st) {
    Stream s{words, base_bits, total_bits, t};
    if (kind == kCodeHuffman)
        decode_sequential_kernel<kCodeHuffman><<<1, 32, 0, st>>>(s, nsym, out_width, out, total_codewords, err);
    else if (kind == kCodeGolombRice)
        decode_sequential_kernel<kCodeGolombRice><<<1, 32, 0, st>>>(s, nsym, out_width, out, total_codewords, err);
    else
        decode_sequential_kernel<kCodeExpGolomb><<<1, 32, 0, st>>>(s, nsym, out_width, out, total_codewords, err);
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
