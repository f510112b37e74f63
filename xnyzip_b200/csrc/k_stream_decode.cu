// Parallel decoding of one unindexed prefix-code stream: Huffman (huffman_encoder.hpp:205-243),
// Golomb-Rice (golomb_rice_encoder.hpp:150-192) and exp-Golomb (huffman_encoder.hpp:398-442).
// The streams carry no sync points, so decoding is exact for any prefix code:
//
//   1. every thread owns one S-bit subsequence and computes, for each entry offset e < L
//      (L = longest codeword; Golomb-Rice: k + 2 classes), where decoding from there leaves
//      the subsequence and how many codewords start inside.  Chains that reach a codeword
//      start of one of R recorded root chains reuse its result (the roots' codeword starts
//      are kept as bitmaps over the first WIN bits);
//   2. warp 0 composes the block's T transition tables;
//   3. blocks resolve their true entry offset by decoupled look-back over the predecessors'
//      composed tables (function composition with warp shuffles);
//   4. lane 0 walks the block's tables from the true entry (entries a table does not cover,
//      after a codeword longer than L crossed a boundary, are decoded on the spot);
//   5. every thread decodes its subsequence once from its true entry and stores the symbols.
//
// The block's stream words (plus a halo) and the Huffman primary table are staged in shared
// memory; codewords are read through a 64-bit register bit buffer refilled one word at a
// time.  Waits are bounded (kSpinLimit): a block that gives up sets kErrTimeout and the
// host's fallback flag and returns.
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int T = kDecodeBlockSubs;     // subsequences (threads) per block
constexpr int HALO = 8;                 // words staged after the block's range
// Subsequence geometry per code: bits per subsequence, staged words per block.
template <int KIND>
struct Geo {
    static constexpr int S = KIND == kCodeGolombRice ? kDecodeSubBitsGR : kDecodeSubBits;
    static constexpr int STAGED = T * S / 32 + HALO;
};
constexpr int WIN = 256;                // root bitmaps cover codeword starts in [0, WIN)
constexpr int WINW = WIN / 32;
constexpr int R = 3;                    // recorded root chains per subsequence
constexpr int kMaxL = kDecodeMaxL;
constexpr int kMaxRootBits = 11;
constexpr u32 kOOD = 0xffu;             // exit outside the next subsequence's entry range
constexpr u64 kFar = 1ull << 20;        // length given to an invalid Huffman code: ends the chain
static_assert(kDecodeSubBits % 32 == 0 && kDecodeSubBitsGR % 32 == 0 && T % 32 == 0 && T <= 1024 &&
                  WIN <= kDecodeSubBits && WIN <= kDecodeSubBitsGR && kDecodeSubBits <= kDecodeSubBitsGR,
              "decode geometry");

// ------------------------------------------------------------- stream source ----------
// A stream starts `base` (< 32) bits into `g`.  Word k of `g` is read from shared memory
// when staged, else from global memory; words past the stream read as zero.
struct Src {
    const u32* g;
    u32 base;
    u64 total_bits;
    u64 nwords;
    const u32* sm;
    u64 sm_w0;
    u64 staged;  // words in sm
    __device__ __forceinline__ u32 word(u64 k) const {
        const u64 d = k - sm_w0;
        if (d < staged) return sm[d];
        return k < nwords ? __ldg(g + k) : 0u;
    }
    __device__ __forceinline__ u32 word_be(u64 k) const { return __byte_perm(word(k), 0, 0x0123); }
    // 32 bits of the MSB-first stream from stream bit p, first bit in bit 31.
    __device__ __forceinline__ u32 msb32(u64 p) const {
        const u64 q = base + p;
        const u32 o = (u32)(q & 31u);
        const u32 a = word_be(q >> 5);
        return o ? ((a << o) | (word_be((q >> 5) + 1) >> (32u - o))) : a;
    }
    // 64 bits of the LSB-first stream from stream bit p, first bit in bit 0.
    __device__ __forceinline__ u64 lsb64(u64 p) const {
        const u64 q = base + p;
        const u32 o = (u32)(q & 31u);
        const u64 k = q >> 5;
        const u64 lo = (u64)word(k) | ((u64)word(k + 1) << 32);
        return o ? ((lo >> o) | ((u64)word(k + 2) << (64u - o))) : lo;
    }
};

// MSB-first bit buffer: the next bit is bit 63 of buf, nb bits are valid, the rest are 0.
struct MsbReader {
    u64 buf;
    int nb;
    u64 wk;
    __device__ __forceinline__ void init(const Src& s, u64 p) {
        const u64 q = s.base + p;
        wk = q >> 5;
        const u32 o = (u32)(q & 31u);
        buf = (((u64)s.word_be(wk) << 32) | (u64)s.word_be(wk + 1)) << o;
        nb = 64 - (int)o;
        wk += 2;
    }
    __device__ __forceinline__ void refill(const Src& s) {
        if (nb <= 32) {
            buf |= (u64)s.word_be(wk) << (32 - nb);
            nb += 32;
            ++wk;
        }
    }
    __device__ __forceinline__ void skip(int n) {
        buf = n >= 64 ? 0ull : buf << n;
        nb -= n;
    }
};

// LSB-first bit buffer: the next bit is bit 0 of buf.
struct LsbReader {
    u64 buf;
    int nb;
    u64 wk;
    __device__ __forceinline__ void init(const Src& s, u64 p) {
        const u64 q = s.base + p;
        wk = q >> 5;
        const u32 o = (u32)(q & 31u);
        buf = ((u64)s.word(wk) | ((u64)s.word(wk + 1) << 32)) >> o;
        nb = 64 - (int)o;
        wk += 2;
    }
    __device__ __forceinline__ void refill(const Src& s) {
        if (nb <= 32) {
            buf |= (u64)s.word(wk) << nb;
            nb += 32;
            ++wk;
        }
    }
    __device__ __forceinline__ void skip(int n) {
        buf = n >= 64 ? 0ull : buf >> n;
        nb -= n;
    }
};

// ------------------------------------------------------------- codewords --------------
struct Code {
    const u32* root;   // primary table (shared memory when staged)
    const u32* tree;   // global
    const u64* symvals;  // null: table entries hold the symbol values themselves
    int rb;
    int k;
    int zigzag;
};

// Huffman from a 32-bit window: primary lookup, tree walk for codes longer than rb.
// Returns the length (0: no code) and the entry payload (symbol value or index).
__device__ __forceinline__ u32 huff_lookup(const Code& c, u32 top, u32& sym) {
    const u32 e = c.root[top >> (32 - c.rb)];
    if (!(e & 0x80000000u)) {
        sym = e & 0xffffffu;
        return e >> 24;
    }
    u32 node = e & 0x7fffffffu;
    for (u32 i = (u32)c.rb; i < 32u; ++i) {
        const u32 ch = __ldg(&c.tree[2 * node + ((top >> (31u - i)) & 1u)]);
        if (ch & 0x80000000u) {
            sym = ch & 0x7fffffffu;
            return ch == 0xffffffffu ? 0u : i + 1;
        }
        node = ch;
    }
    sym = 0;
    return 0;
}

// Golomb-Rice codeword at stream bit p without the bit buffer (long runs, large k).
// A codeword that does not end inside the stream returns total_bits + 1 - p.
__device__ u64 gr_generic(const Src& s, u64 p, int k, u64& val) {
    u64 q = 0;
    u64 v = s.lsb64(p);
    while (v == ~0ull) {
        q += 64;
        if (p + q >= s.total_bits + 64) {
            val = 0;
            return s.total_bits + 1 - p;
        }
        v = s.lsb64(p + q);
    }
    q += (u64)(__ffsll((long long)~v) - 1);
    if (p + q + 1 + (u64)k > s.total_bits) {
        val = 0;
        return s.total_bits + 1 - p;
    }
    const u64 r = k ? (s.lsb64(p + q + 1) & ((1ull << k) - 1)) : 0ull;
    val = (q << k) + r;
    return q + 1 + (u64)k;
}

// exp-Golomb codeword at stream bit p without the bit buffer.
__device__ u64 eg_generic(const Src& s, u64 p, int k, int zigzag, u64& val) {
    u64 z = 0;
    u32 w = s.msb32(p);
    while (w == 0u) {
        z += 32;
        if (p + z >= s.total_bits + 64) {
            val = 0;
            return s.total_bits + 1 - p;
        }
        w = s.msb32(p + z);
    }
    z += (u64)__clz((int)w);
    if (p + 2 * z + 1 + (u64)k > s.total_bits) {
        val = 0;
        return s.total_bits + 1 - p;
    }
    u64 n1;
    if (z + 1 <= 32) {
        n1 = s.msb32(p + z) >> (31 - z);
    } else {
        const u64 hi = s.msb32(p + z), lo = s.msb32(p + z + 32);
        n1 = z + 1 >= 64 ? ~0ull : (((hi << 32) | lo) >> (63 - z));
    }
    const u64 rbits = k ? (s.msb32(p + 2 * z + 1) >> (32 - k)) : 0ull;
    const u64 low = k ? (u64)(__brev((u32)rbits) >> (32 - k)) : 0ull;
    const u64 u = ((n1 - 1) << k) | low;
    val = zigzag ? ((u >> 1) ^ (~(u & 1ull) + 1ull)) : u;
    return 2 * z + 1 + (u64)k;
}

// One codeword through the bit buffer at stream bit p (the reader is positioned at p).
// Returns the length; Huffman returns kFar for a prefix that is no code.  `val` is the
// symbol value (Huffman: the table payload, mapped through symvals when present).
template <int KIND>
struct Dec;

template <>
struct Dec<kCodeHuffman> {
    MsbReader r;
    __device__ __forceinline__ void init(const Src& s, u64 p) { r.init(s, p); }
    __device__ __forceinline__ u64 step(const Src& s, const Code& c, u64, u64& val, bool want) {
        r.refill(s);
        u32 sym;
        const u32 len = huff_lookup(c, (u32)(r.buf >> 32), sym);
        if (!len) {
            val = 0;
            return kFar;
        }
        r.skip((int)len);
        if (want) val = c.symvals ? __ldg(&c.symvals[sym]) : (u64)sym;
        return len;
    }
};

template <>
struct Dec<kCodeGolombRice> {
    LsbReader r;
    __device__ __forceinline__ void init(const Src& s, u64 p) { r.init(s, p); }
    __device__ __forceinline__ u64 step(const Src& s, const Code& c, u64 p, u64& val, bool) {
        r.refill(s);
        const int k = c.k;
        if (r.buf != ~0ull) {
            const int t = __ffsll((long long)~r.buf) - 1;
            if (t < r.nb && t + 1 + k <= r.nb) {
                const u64 rem = k ? ((r.buf >> (t + 1)) & ((1ull << k) - 1)) : 0ull;
                val = ((u64)t << k) | rem;
                const int len = t + 1 + k;
                r.skip(len);
                return (u64)len;
            }
        }
        const u64 len = gr_generic(s, p, k, val);
        r.init(s, p + len);
        return len;
    }
};

template <>
struct Dec<kCodeExpGolomb> {
    MsbReader r;
    __device__ __forceinline__ void init(const Src& s, u64 p) { r.init(s, p); }
    __device__ __forceinline__ u64 step(const Src& s, const Code& c, u64 p, u64& val, bool) {
        r.refill(s);
        const int k = c.k;
        if (r.buf) {
            const int z = __clzll((long long)r.buf);
            const int len = 2 * z + 1 + k;
            if (z < r.nb && len <= r.nb) {
                const u64 n1 = (r.buf << z) >> (63 - z);
                const u64 rbits = k ? ((r.buf << (2 * z + 1)) >> (64 - k)) : 0ull;
                const u64 low = k ? (u64)(__brev((u32)rbits) >> (32 - k)) : 0ull;
                const u64 u = ((n1 - 1) << k) | low;
                val = c.zigzag ? ((u >> 1) ^ (~(u & 1ull) + 1ull)) : u;
                r.skip(len);
                return (u64)len;
            }
        }
        const u64 len = eg_generic(s, p, k, c.zigzag, val);
        r.init(s, p + len);
        return len;
    }
};

// One codeword at p without a persistent reader (the on-the-spot walks of step 4).
template <int KIND>
__device__ __forceinline__ u64 codeword_at(const Src& s, const Code& c, u64 p, u64& val) {
    Dec<KIND> d;
    d.init(s, p);
    return d.step(s, c, p, val, false);
}

// One-bits of an LSB-first stream from stream bit p up to the first zero.
__device__ u64 lead_ones(const Src& s, u64 p) {
    u64 q = 0;
    while (p + q < s.total_bits) {
        const u64 v = s.lsb64(p + q);
        if (v != ~0ull) return q + (u64)(__ffsll((long long)~v) - 1);
        q += 64;
    }
    return q;
}

// Entry classes.  Golomb-Rice: a codeword crossing into subsequence s ends at an offset
// x <= k, or its terminating zero lies inside s after a run of ones that reaches back to
// s's first bit, so x = k + 1 + (leading ones of s): k + 2 classes, the last one "special".
// Other codes: offsets 0 .. L-1.
template <int KIND>
__device__ __forceinline__ u32 entry_index(u64 x, int L, int k) {
    if (KIND == kCodeGolombRice) return x <= (u64)k ? (u32)x : (u32)(k + 1);
    return x < (u64)L ? (u32)x : kOOD;
}
template <int KIND>
__device__ __forceinline__ u64 entry_offset(const Src& s, u32 i, u64 Bsub, int k) {
    if (KIND == kCodeGolombRice && i == (u32)(k + 1)) return (u64)k + 1 + lead_ones(s, Bsub);
    return i;
}

// Golomb-Rice transition table of one subsequence [B, Bend) by lockstep simulation.  The
// codeword-start map f(s) = z(s) + 1 + k (z(s): first zero bit at or after s) is monotone, so
// the chains of entries 0..k keep their order, merge when they land on one position, and at
// step n all lie within codeword n of entry 0's chain.  While that codeword is shorter than
// 64 bits (k <= 30 and a unary part below 64 - k - 1 bits), the active chains are a 64-bit
// position mask over a shared 128-bit zero window, and their entries a boundary mask over
// 0..k.  Entry k + 1 (a unary run crossing B) is entry 0's chain after its first codeword.
// Called by every thread of the warp (valid: this thread owns a subsequence); the loops are
// warp-uniform (__any_sync) so that lanes with different chain counts stay converged.
// Returns false (table incomplete) when a codeword is too long for the masks or the stream
// ends within reach; the caller then runs the generic loop.
__device__ bool gr_lockstep_table(const Src& src, u64 B, u64 Bend, int k, u32* tab, int t, bool valid) {
    constexpr int S = Geo<kCodeGolombRice>::S;
    const u32 span = valid ? (u32)(Bend - B) : 0u;
    const bool full = span == (u32)S;
    // near the end of the stream codewords may run past it (the generic decoder gives those
    // a length that ends the chain): left to the generic loop
    bool ok = valid && B + span + 192 <= src.total_bits;
    const int ne = min(k + 1, (int)span);  // entries with a codeword start inside
    if (ok)
        for (int e = ne; e <= k; ++e) tab[e * T + t] = kOOD;  // (only in a short last subsequence)
    u64 act = ok ? (ne >= 64 ? ~0ull : ((1ull << ne) - 1ull)) : 0ull;  // group positions - base
    u64 gb = act;     // first entry of every group
    u64 alive = act;  // entries not yet recorded
    u32 base = 0, n = 0, exit0 = kOOD, count0 = 0;
    // The 128 bits from B + base, kept in five stream words that move forward with base (the
    // groups only advance), instead of two six-word reads per step.
    u64 wk = (src.base + B) >> 5;
    u32 wv[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) wv[i] = src.word(wk + i);
    while (__any_sync(kFullMask, act != 0ull)) {
        u64 z0 = 0, z1 = 0;
        if (act) {
            const u64 q = src.base + B + base;
            const u64 kk = q >> 5;
            if (kk - wk >= 5) {
                wk = kk;
#pragma unroll
                for (int i = 0; i < 5; ++i) wv[i] = src.word(wk + i);
            } else {
                while (wk < kk) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) wv[i] = wv[i + 1];
                    wv[4] = src.word(wk + 5);
                    ++wk;
                }
            }
            const u32 o = (u32)(q & 31u);
            const u64 a = (u64)wv[0] | ((u64)wv[1] << 32), b = (u64)wv[2] | ((u64)wv[3] << 32);
            z0 = ~(o ? (a >> o) | (b << (64u - o)) : a);
            z1 = ~(o ? (b >> o) | ((u64)wv[4] << (64u - o)) : b);
            ++n;
        }
        // successors, in order; groups landing on the previous group's position merge
        u64 a = act, g = gb, nact = 0, ngb = gb;
        u32 first_s = 0, prev_s = 0xffffffffu;
        bool any = false;
        while (__any_sync(kFullMask, a != 0ull)) {
            if (!a) continue;
            const int j = __ffsll((long long)a) - 1;
            a &= a - 1;
            const int e0 = __ffsll((long long)g) - 1;
            g &= g - 1;
            u32 zp = 0;
            if (z0 >> j) {
                zp = base + (u32)j + (u32)(__ffsll((long long)(z0 >> j)) - 1);
            } else if (z1) {
                zp = base + 64u + (u32)(__ffsll((long long)z1) - 1);
            } else {  // a unary run longer than the window
                ok = false;
                a = 0;
                continue;
            }
            const u32 sp = zp + 1u + (u32)k;
            if (sp == prev_s) {
                ngb &= ~(1ull << e0);
                continue;
            }
            if (!any) {
                first_s = sp;
                any = true;
            }
            if (sp - first_s >= 64u) {  // the chains span more than 64 bits
                ok = false;
                a = 0;
                continue;
            }
            nact |= 1ull << (sp - first_s);
            prev_s = sp;
        }
        if (!ok) {
            act = 0;
            continue;
        }
        if (!act) continue;
        act = nact;
        gb = ngb;
        base = first_s;
        // groups at or past the end leave: they are the top groups, entries from their first
        // entry up to the next group's first entry (or the last alive entry)
        const u32 lo = span > base ? span - base : 0u;  // first leaving bit
        const u64 leave = lo >= 64 ? 0ull : (act >> lo) << lo;
        if (leave) {
            u64 a2 = act, g2 = gb;
            while (a2) {
                const int j = __ffsll((long long)a2) - 1;
                a2 &= a2 - 1;
                const int e0 = __ffsll((long long)g2) - 1;
                g2 &= g2 - 1;
                if (!((leave >> j) & 1ull)) continue;
                const int e1 = g2 ? __ffsll((long long)g2) - 1 : 64;  // next group's first entry
                const u32 P = base + (u32)j;
                const u32 ox = full ? entry_index<kCodeGolombRice>((u64)P - S, k + 2, k) : kOOD;
                const u64 below1 = e1 >= 64 ? ~0ull : ((1ull << e1) - 1ull), below0 = (1ull << e0) - 1ull;
                u64 m = alive & below1 & ~below0;
                while (m) {
                    const int e = __ffsll((long long)m) - 1;
                    m &= m - 1;
                    tab[e * T + t] = ox | (n << 8);
                    if (e == 0) {
                        exit0 = ox;
                        count0 = n;
                    }
                }
                alive &= ~below1 | below0;
            }
            act &= ~leave;
            gb &= alive;
        }
    }
    if (ok) tab[(k + 1) * T + t] = exit0 | ((count0 - 1u) << 8);
    return ok;
}

struct Args {
    const u32* words;
    u32 base;
    u64 total_bits;
    u64 nsub;
    int L;
    Code code;
    const u32* root_global;
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

// Shared memory: scount[T] u64 | sw[STAGED] | bm[R][WINW][T] | sstart[T] | slot | tab[L][T] | root[2^rb]
template <int KIND>
__host__ __device__ constexpr size_t smem_for(int L, int rb) {
    return 8 * T + 4 * (Geo<KIND>::STAGED + R * WINW * T + T + 4) + 4ull * L * T + (rb ? 4ull << rb : 0);
}

// Output of symbols: u8 streams pack four symbols per 32-bit store where a word lies inside
// the thread's range.
struct ByteOut {
    u8* out;
    u64 first;
    u32 acc;
    __device__ __forceinline__ void put(u64 i, u64 v) {
        const u32 sh = (u32)(i & 3u) * 8u;
        acc = (sh ? acc : 0u) | ((u32)(v & 0xffu) << sh);
        if (sh == 24u) {
            const u64 w0 = i & ~3ull;
            if (w0 >= first) {
                *reinterpret_cast<u32*>(out + w0) = acc;
            } else {
                for (u64 j = first; j <= i; ++j) out[j] = (u8)(acc >> ((j & 3u) * 8u));
            }
        }
    }
    __device__ __forceinline__ void flush(u64 end) {  // symbols [.., end) were put
        if (end & 3u) {
            const u64 w0 = end & ~3ull;
            for (u64 j = w0 > first ? w0 : first; j < end; ++j) out[j] = (u8)(acc >> ((j & 3u) * 8u));
        }
    }
};

template <int KIND>
__global__ void __launch_bounds__(T) decode_stream_kernel(Args a) {
    constexpr int S = Geo<KIND>::S;
    constexpr int STAGED = Geo<KIND>::STAGED;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    u64* scount = reinterpret_cast<u64*>(smem_raw);
    u32* sw = reinterpret_cast<u32*>(scount + T);
    u32* bm = sw + STAGED;
    u32* sstart = bm + R * WINW * T;
    u32* slotp = sstart + T;
    u32* tab = slotp + 4;
    u32* sroot = tab + (size_t)a.L * T;

    const u32 tile = claim_tile(a.tile_counter, slotp);
    const int t = threadIdx.x;
    const u64 first_sub = (u64)tile * T;
    const u32 nvalid = (u32)min((u64)T, a.nsub - first_sub);
    const int gk = a.code.k;
    const int L = a.L;

    Src src;
    src.g = a.words;
    src.base = a.base;
    src.total_bits = a.total_bits;
    src.nwords = (a.base + a.total_bits + 31) >> 5;
    src.sm = sw;
    src.sm_w0 = first_sub * (S / 32);
    src.staged = STAGED;
    for (int i = t; i < STAGED; i += T) {
        const u64 k = src.sm_w0 + i;
        sw[i] = k < src.nwords ? __ldg(a.words + k) : 0u;
    }
    Code code = a.code;
    if (KIND == kCodeHuffman) {
        for (int i = t; i < (1 << code.rb); i += T) sroot[i] = __ldg(a.root_global + i);
        code.root = sroot;
    }
    __syncthreads();

    const u64 B = (first_sub + t) * (u64)S;
    const u64 Bend = min(B + S, a.total_bits);

    // ---- 1. transition table of my subsequence ----
    bool done1 = false;
    if (KIND == kCodeGolombRice && gk <= 30) done1 = gr_lockstep_table(src, B, Bend, gk, tab, t, (u32)t < nvalid);
    if ((u32)t < nvalid && !done1) {
        u32 rx[R] = {}, rc[R] = {};
        int nroots = 0;
        auto bmw = [&](int r, int w) -> u32& { return bm[(r * WINW + w) * T + t]; };
        auto popc_below = [&](int r, u32 q) {
            u32 c = 0;
            for (u32 w = 0; w < (q >> 5); ++w) c += __popc(bmw(r, (int)w));
            if (q & 31u) c += __popc(bmw(r, (int)(q >> 5)) & ((1u << (q & 31u)) - 1u));
            return c;
        };
        for (int e = 0; e < L; ++e) {
            const u64 off = entry_offset<KIND>(src, (u32)e, B, gk);
            u64 p = B + off;
            u32 ox = kOOD, oc = 0;
            if (p >= Bend) {  // no codeword starts here: the entry passes through
                ox = Bend == B + S ? entry_index<KIND>(off - S, L, gk) : kOOD;
                tab[e * T + t] = ox;
                continue;
            }
            int hit = -1;
            if (off < (u64)WIN) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r < nroots && ((bmw(r, (int)(off >> 5)) >> (off & 31u)) & 1u)) hit = r;
            }
            if (hit >= 0) {
#pragma unroll
                for (int r = 0; r < R; ++r)
                    if (r == hit) {
                        ox = rx[r];
                        oc = rc[r];
                    }
                oc -= popc_below(hit, (u32)off);
                tab[e * T + t] = ox | (oc << 8);
                continue;
            }
            const bool rec = nroots < R && off < (u64)WIN;
            if (rec)
                for (int w = 0; w < WINW; ++w) bmw(nroots, w) = 0u;
            int cw = (int)(off >> 5);
            u32 cbits = rec ? (1u << (off & 31u)) : 0u;
            u32 rw[R];
#pragma unroll
            for (int r = 0; r < R; ++r) rw[r] = (r < nroots && off < (u64)WIN) ? bmw(r, cw) : 0u;
            Dec<KIND> d;
            d.init(src, p);
            u32 c = 0;
            bool merged = false;
            while (p < Bend) {
                u64 v;
                p += d.step(src, code, p, v, false);
                ++c;
                if (p < Bend && p - B < (u64)WIN) {
                    const u32 q = (u32)(p - B);
                    const int w = (int)(q >> 5);
                    if (w != cw) {
                        if (rec) bmw(nroots, cw) = cbits;
                        cbits = 0u;
                        cw = w;
#pragma unroll
                        for (int r = 0; r < R; ++r) rw[r] = r < nroots ? bmw(r, w) : 0u;
                    }
                    const u32 bit = 1u << (q & 31u);
                    int h = -1;
                    u32 hx = 0, hc = 0;
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (r < nroots && (rw[r] & bit)) {
                            h = r;
                            hx = rx[r];
                            hc = rc[r];
                        }
                    if (h >= 0) {
                        merged = true;
                        ox = hx;
                        oc = c + hc - popc_below(h, q);
                        break;
                    }
                    cbits |= bit;
                }
            }
            if (!merged) {
                if (rec && cw < WINW) bmw(nroots, cw) = cbits;
                ox = (Bend == B + S && p >= Bend) ? entry_index<KIND>(p - (B + S), L, gk) : kOOD;
                oc = c;
                if (rec) {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        if (r == nroots) {
                            rx[r] = ox;
                            rc[r] = c;
                        }
                    ++nroots;
                }
            }
            tab[e * T + t] = ox | (oc << 8);
        }
    }
    __syncthreads();

    // ---- 2. composed table of the block (warp 0; lane holds entries lane and lane + 32) ----
    // ---- 3. look-back over predecessor blocks ----
    // ---- 4. true entry of every subsequence ----
    if (t < 32) {
        u32 gx[2];
        u64 gc[2];
        for (int h = 0; h < 2; ++h) {
            const int e = t + 32 * h;
            u32 x = e < L ? (u32)e : kOOD;
            u64 c = 0;
            for (u32 j = 0; j < nvalid && x != kOOD; ++j) {
                const u32 v = tab[x * T + j];
                c += v >> 8;
                x = v & 0xffu;
            }
            gx[h] = x;
            gc[h] = c;
        }
        u64 E = 0, C = 0;
        bool failed = false;
        if (tile > 0) {
            for (int h = 0; h < 2; ++h) st_volatile(&a.agg[(u64)tile * kMaxL + t + 32 * h], (u64)gx[h] | (gc[h] << 8));
            __threadfence();
            __syncwarp();
            if (t == 0) st_volatile(&a.flag[tile], 1u);
            // G: composition of the aggregates walked so far (identity to start).
            u32 Gx[2] = {(u32)t, (u32)t + 32};
            u64 Gc[2] = {0, 0};
            long long pidx = (long long)tile - 1;
            u32 spins = 0;
            bool need_pred = false;
            while (true) {
                u32 f = 0;
                if (t == 0) f = ld_volatile(&a.flag[pidx]);
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
                    const u64 X = ld_volatile(&a.inc[(u64)pidx * 2]);
                    const u64 CX = ld_volatile(&a.inc[(u64)pidx * 2 + 1]);
                    if (pidx == (long long)tile - 1) {  // exact entry from the direct predecessor
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
                // aggregate F of block pidx: G <- G o F (both halves read G before either is
                // overwritten)
                u32 nx[2];
                u64 nc[2];
                for (int h = 0; h < 2; ++h) {
                    const u64 fv = ld_volatile(&a.agg[(u64)pidx * kMaxL + t + 32 * h]);
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
                --pidx;
                if (pidx < 0) {  // cannot happen: tile 0 always publishes its inclusive value
                    failed = true;
                    break;
                }
            }
            if (need_pred && !failed) {
                // wait for the direct predecessor's exact exit
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
        // (E is an entry index when it came from a composed table, an offset when it came
        // from a predecessor's walk; entry_index maps both.)
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
            if (KIND == kCodeGolombRice && E > (u64)gk) x = entry_offset<KIND>(src, (u32)(gk + 1), first_sub * S, gk);
            u64 c = C;
            for (u32 j = 0; j < nvalid; ++j) {
                sstart[j] = (u32)min(x, (u64)0xffffffffu);
                scount[j] = c;
                const u32 xi = entry_index<KIND>(x, L, gk);
                const u32 v = xi != kOOD ? tab[xi * T + j] : kOOD;
                if ((v & 0xffu) != kOOD) {
                    c += v >> 8;
                    x = entry_offset<KIND>(src, v & 0xffu, (first_sub + j + 1) * S, gk);
                } else {
                    const u64 Bj = (first_sub + j) * S;
                    const u64 Ej = min(Bj + S, a.total_bits);
                    u64 pp = Bj + x;
                    if (pp < Ej) {
                        Dec<KIND> d;
                        d.init(src, pp);
                        while (pp < Ej) {
                            u64 val;
                            pp += d.step(src, code, pp, val, false);
                            ++c;
                        }
                    }
                    x = pp >= Bj + S ? pp - (Bj + S) : 0ull;
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
    if ((u32)t < nvalid && !(*(volatile u32*)a.need_fallback)) {
        u64 idx = scount[t];
        u64 p = B + sstart[t];
        if (p < Bend && idx < a.nsym) {
            Dec<KIND> d;
            d.init(src, p);
            if (a.out_width == 1) {
                ByteOut bo{static_cast<u8*>(a.out), idx, 0u};
                while (p < Bend && idx < a.nsym) {
                    u64 v;
                    const u64 len = d.step(src, code, p, v, true);
                    if (p + len > a.total_bits) {
                        atomicOr(a.err, kErrBadStream);
                        break;
                    }
                    bo.put(idx, v);
                    ++idx;
                    p += len;
                }
                bo.flush(idx);
            } else {
                while (p < Bend && idx < a.nsym) {
                    u64 v;
                    const u64 len = d.step(src, code, p, v, true);
                    if (p + len > a.total_bits) {
                        atomicOr(a.err, kErrBadStream);
                        break;
                    }
                    if (a.out_width == 4) static_cast<u32*>(a.out)[idx] = (u32)v;
                    else static_cast<u64*>(a.out)[idx] = v;
                    ++idx;
                    p += len;
                }
            }
        }
    }
}

// One-thread decoder, run by the host after a bounded wait of the parallel decoder expired.
template <int KIND>
__global__ void decode_sequential_kernel(Args a) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Src src;
    src.g = a.words;
    src.base = a.base;
    src.total_bits = a.total_bits;
    src.nwords = (a.base + a.total_bits + 31) >> 5;
    src.sm = nullptr;
    src.sm_w0 = 0;
    src.staged = 0;  // nothing staged
    Code code = a.code;
    code.root = a.root_global;
    u64 p = 0, i = 0;
    Dec<KIND> d;
    d.init(src, 0);
    while (i < a.nsym && p < a.total_bits) {
        u64 v;
        const u64 len = d.step(src, code, p, v, true);
        if (p + len > a.total_bits) {
            atomicOr(a.err, kErrBadStream);
            break;
        }
        if (a.out_width == 1) static_cast<u8*>(a.out)[i] = (u8)v;
        else if (a.out_width == 4) static_cast<u32*>(a.out)[i] = (u32)v;
        else static_cast<u64*>(a.out)[i] = v;
        ++i;
        p += len;
    }
    *a.total_codewords = i;
}

// A Huffman stream whose codewords all have one length `len` (<= kMaxRootBits): symbol i is
// bits [i len, (i + 1) len) of the stream, one primary-table lookup each, so the stream needs
// neither entry tables nor look-back.  Thread g decodes symbols 4g .. 4g + 3 from one 64-bit
// window (4 len <= 44 bits) and stores u8 symbols four at a time.  A chunk that is no
// codeword sets kErrBadStream, as the chained decoder does.
__global__ void __launch_bounds__(256) decode_fixed_kernel(const u32* __restrict__ words, u32 base, u64 nwords,
                                                           int len, const u32* __restrict__ root,
                                                           const u64* __restrict__ symvals, u64 nsym, int width,
                                                           void* out, bool packed_ok, u32* err,
                                                           unsigned long long* sum_out) {
    const u64 groups = (nsym + 3) / 4;
    u64 sum = 0;  // sum_out: the sum of max(symbol, 0) over 32-bit symbols (the -rle point count)
    auto wbe = [&](u64 k) -> u64 { return k < nwords ? (u64)__byte_perm(__ldg(words + k), 0, 0x0123) : 0ull; };
    for (u64 g = (u64)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += (u64)gridDim.x * blockDim.x) {
        const u64 i0 = 4 * g;
        const int cnt = (int)min((u64)4, nsym - i0);
        const u64 q = (u64)base + i0 * (u64)len;
        const u64 k = q >> 5;
        const u32 o = (u32)(q & 31u);
        u64 win = ((wbe(k) << 32) | wbe(k + 1)) << o;
        if (o) win |= wbe(k + 2) >> (32u - o);
        bool bad = false;
        u32 packed = 0;
        for (int j = 0; j < cnt; ++j) {
            const u32 code = (u32)(win >> (64 - len));
            win <<= len;
            const u32 e = __ldg(root + code);
            if ((e >> 24) != (u32)len) bad = true;
            const u64 val = symvals ? __ldg(symvals + (e & 0xffffffu)) : (u64)(e & 0xffffffu);
            if (width == 1) {
                packed |= ((u32)val & 0xffu) << (8 * j);
            } else {
                reinterpret_cast<u32*>(out)[i0 + j] = (u32)val;
                sum += (u64)max((i32)(u32)val, 0);
            }
        }
        if (width == 1) {
            u8* o8 = reinterpret_cast<u8*>(out) + i0;
            if (cnt == 4 && packed_ok) {
                *reinterpret_cast<u32*>(o8) = packed;
            } else {
                for (int j = 0; j < cnt; ++j) o8[j] = (u8)(packed >> (8 * j));
            }
        }
        if (bad) atomicOr(err, kErrBadStream);
    }
    if (sum_out) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(kFullMask, sum, d);
        if ((threadIdx.x & 31u) == 0 && sum) atomicAdd(sum_out, sum);
    }
}

__global__ void flag_error_kernel(u32* err) { atomicOr(err, kErrBadStream); }
void atomic_flag_host_error(u32* err, cudaStream_t st) { flag_error_kernel<<<1, 1, 0, st>>>(err); }

Args make_args(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits, const DecodeTable& t, int L,
               uint64_t nsym, int out_width, void* out) {
    Args a{};
    a.words = words;
    a.base = (u32)base_bits;
    a.total_bits = total_bits;
    const u64 S = kind == kCodeGolombRice ? (u64)kDecodeSubBitsGR : (u64)kDecodeSubBits;
    a.nsub = (total_bits + S - 1) / S;
    a.L = kind == kCodeGolombRice ? (t.param + 2 < kMaxL ? t.param + 2 : kMaxL) : (L < 1 ? 1 : (L > kMaxL ? kMaxL : L));
    a.code.root = t.root;
    a.code.tree = t.tree;
    a.code.symvals = t.symvals;
    a.code.rb = kind == kCodeHuffman ? t.root_bits : 0;
    a.code.k = t.param;
    a.code.zigzag = t.zigzag;
    a.root_global = t.root;
    a.nsym = nsym;
    a.out_width = out_width;
    a.out = out;
    return a;
}

}  // namespace

void launch_decode_stream(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits, DecodeTable t,
                          int L, const uint32_t* L_run, uint64_t nsym, int out_width, void* out, uint32_t* flag,
                          unsigned long long* agg, unsigned long long* inc, uint32_t* tile_counter, uint32_t* err,
                          uint32_t* need_fallback, unsigned long long* total_codewords, cudaStream_t st) {
    (void)L_run;
    if (kind == kCodeHuffman && (t.root_bits < 1 || t.root_bits > kMaxRootBits)) {
        atomic_flag_host_error(err, st);  // the host builds tables with 1 <= root_bits <= 11
        return;
    }
    Args a = make_args(kind, words, base_bits, total_bits, t, L, nsym, out_width, out);
    a.flag = flag;
    a.agg = agg;
    a.inc = inc;
    a.tile_counter = tile_counter;
    a.err = err;
    a.need_fallback = need_fallback;
    a.total_codewords = total_codewords;
    const unsigned tiles = (unsigned)((a.nsub + T - 1) / T);
    if (!tiles) return;
    // The launch uses what this stream needs; the function's limit is always set to the
    // largest size any stream can need (the same value from every thread, so concurrent
    // launches from other contexts cannot lower it between this call and the launch).
    const int smem = kind == kCodeGolombRice ? (int)smem_for<kCodeGolombRice>(a.L, a.code.rb)
                                             : (int)smem_for<kCodeHuffman>(a.L, a.code.rb);
    const int smem_max = kind == kCodeGolombRice ? (int)smem_for<kCodeGolombRice>(kMaxL, kMaxRootBits)
                                                 : (int)smem_for<kCodeHuffman>(kMaxL, kMaxRootBits);
    if (kind == kCodeHuffman) {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeHuffman>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
        decode_stream_kernel<kCodeHuffman><<<tiles, T, smem, st>>>(a);
    } else if (kind == kCodeGolombRice) {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeGolombRice>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem_max);
        decode_stream_kernel<kCodeGolombRice><<<tiles, T, smem, st>>>(a);
    } else {
        cudaFuncSetAttribute(decode_stream_kernel<kCodeExpGolomb>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem_max);
        decode_stream_kernel<kCodeExpGolomb><<<tiles, T, smem, st>>>(a);
    }
}

void launch_decode_fixed(const uint32_t* words, uint64_t base_bits, uint64_t total_bits, DecodeTable t, int len,
                         uint64_t nsym, int out_width, void* out, uint32_t* err, cudaStream_t st,
                         unsigned long long* sum_out) {
    if (!nsym) return;
    if (len < 1 || len > kMaxRootBits || len != t.root_bits || (out_width != 1 && out_width != 4) ||
        nsym * (uint64_t)len > total_bits) {
        atomic_flag_host_error(err, st);  // the host only routes complete fixed-length streams here
        return;
    }
    const u64 nwords = (base_bits + total_bits + 31) / 32;
    u64 blocks = (nsym / 4 + 256) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    const bool packed_ok = (reinterpret_cast<uintptr_t>(out) & 3u) == 0;
    decode_fixed_kernel<<<(unsigned)blocks, 256, 0, st>>>(words, (u32)base_bits, nwords, len, t.root, t.symvals, nsym,
                                                          out_width, out, packed_ok, err,
                                                          out_width == 4 ? sum_out : nullptr);
}

void launch_decode_sequential(int kind, const uint32_t* words, uint64_t base_bits, uint64_t total_bits,
                              DecodeTable t, uint64_t nsym, int out_width, void* out,
                              unsigned long long* total_codewords, uint32_t* err, cudaStream_t st) {
    Args a = make_args(kind, words, base_bits, total_bits, t, kMaxL, nsym, out_width, out);
    a.err = err;
    a.total_codewords = total_codewords;
    if (kind == kCodeHuffman)
        decode_sequential_kernel<kCodeHuffman><<<1, 32, 0, st>>>(a);
    else if (kind == kCodeGolombRice)
        decode_sequential_kernel<kCodeGolombRice><<<1, 32, 0, st>>>(a);
    else
        decode_sequential_kernel<kCodeExpGolomb><<<1, 32, 0, st>>>(a);
}

}  // namespace dev
}  // namespace xnyz
