// Block-parameter coding of the repos / SFC-delta stream (the extended container).
//
// The stream of n u64 values is cut into blocks of 1024.  Block b is coded with a PFor slot
// width w_b in 0..32 and a Golomb-Rice parameter k_b in 0..31.  Its payload (LSB-first bits,
// starting at the block's bit offset) has four regions:
//   S  1024 slots of w_b bits: slot = v if v < 2^w - 1, else the escape 2^w - 1 (w = 0:
//      every value escapes);
//   U  for each escaping value in order, with e = v - (2^w - 1) and q = e >> k: min(q, 32)
//      one bits and a zero (q >= 32 marks a capped escape);
//   R  for each escaping value, the k low bits of e;
//   X  for each capped escape, the 64 bits of e.
// cost(w, k) = n_b * w + sum over escapes of (min(q, 32) + 1 + k + (q >= 32 ? 64 : 0)) bits.
// Blocks carry their bit offset, so they encode and decode independently, and every region
// decodes warp-parallel (escape j's unary part lies between the (j-1)-th and j-th zero of U).
//
// Kernels (one warp per block): features for the parameter predictor, the exhaustive search
// over all 33 x 32 (w, k) pairs (training labels, fallback and the yardstick of the size
// penalty), the cost of given pairs, the encoder and the decoder.
#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int BLK = kParamBlock;  // values per block
constexpr int PER_LANE = BLK / 32;
constexpr int WARPS = 4;          // warps (blocks) per CTA

__device__ __forceinline__ u64 escape_threshold(int w) { return (1ull << w) - 1ull; }

__device__ __forceinline__ u32 esc_len(u64 e, int k) {
    const u64 q = e >> k;
    return q < 32 ? (u32)q + 1u + (u32)k : 97u + (u32)k;
}

__device__ __forceinline__ u32 block_count(u64 n, u64 b) {
    const u64 s = b * BLK;
    return (u32)min((u64)BLK, n - s);
}

// ------------------------------------------------------------------ features ------------
// f[0..31]: fraction of values with min(31, bitlen(v)) == i; f[32], f[33]: mean and max of
// log2(v + 1), divided by 64.
__global__ void __launch_bounds__(32 * WARPS) features_kernel(const u64* __restrict__ v, u64 n, u64 nblk,
                                                              float* __restrict__ feats) {
    __shared__ u32 hist[WARPS][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b = (u64)blockIdx.x * WARPS + w;
    hist[w][lane] = 0;
    __syncwarp();
    if (b >= nblk) return;
    const u32 cnt = block_count(n, b);
    const u64* p = v + b * BLK;
    float lsum = 0.f, lmax = 0.f;
    for (u32 i = lane; i < cnt; i += 32) {
        const u64 x = p[i];
        const u32 bl = min(31u, bitlen64(x));
        atomicAdd(&hist[w][bl], 1u);
        const float l = log2f(__ull2float_rn(x) + 1.0f);
        lsum += l;
        lmax = fmaxf(lmax, l);
    }
    for (int d = 16; d > 0; d >>= 1) {
        lsum += __shfl_xor_sync(kFullMask, lsum, d);
        lmax = fmaxf(lmax, __shfl_xor_sync(kFullMask, lmax, d));
    }
    __syncwarp();
    float* f = feats + b * kParamFeatures;
    const float inv = 1.0f / (float)cnt;
    f[lane] = (float)hist[w][lane] * inv;
    if (lane == 0) {
        f[32] = lsum * inv * (1.0f / 64.0f);
        f[33] = lmax * (1.0f / 64.0f);
    }
}

// ------------------------------------------------------------------ search --------------
// For each w: escapes e with L = bitlen(e) contribute (1 + k) for k >= L, (e >> k) + 1 + k
// for L - 5 <= k < L, and 97 + k for k < L - 5.  Lanes accumulate the exact middle terms in
// their own shared-memory row and the two others through a histogram of L.
struct SearchShared {
    u32 acc[WARPS][32][33];   // [warp][lane][k] exact middle terms
    u32 hl[WARPS][32][66];    // [warp][lane][L] escapes per bit length
    u32 hs[WARPS][66];        // [warp][L] summed over lanes
    u32 cost[WARPS][33][32];  // [warp][w][k]
};

__global__ void __launch_bounds__(32 * WARPS) search_kernel(const u64* __restrict__ v, u64 n, u64 nblk,
                                                            const u8* __restrict__ only, u8* __restrict__ wout,
                                                            u8* __restrict__ kout, u32* __restrict__ cost_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SearchShared& sh = *reinterpret_cast<SearchShared*>(smem_raw);
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b = (u64)blockIdx.x * WARPS + wi;
    if (b >= nblk) return;
    if (only && !only[b]) return;
    const u32 cnt = block_count(n, b);
    u64 x[PER_LANE];
#pragma unroll
    for (int r = 0; r < PER_LANE; ++r) {
        const u32 i = (u32)r * 32 + lane;
        x[r] = i < cnt ? v[b * BLK + i] : 0ull;
    }
    u32* acc = sh.acc[wi][lane];
    u32* hl = sh.hl[wi][lane];
    for (int w = 0; w <= 32; ++w) {
        for (int k = 0; k < 32; ++k) acc[k] = 0;
        for (int L = 0; L < 66; ++L) hl[L] = 0;
        const u64 thr = escape_threshold(w);
#pragma unroll
        for (int r = 0; r < PER_LANE; ++r) {
            const u32 i = (u32)r * 32 + lane;
            if (i >= cnt || x[r] < thr) continue;
            const u64 e = x[r] - thr;
            const int L = (int)bitlen64(e);
            hl[L] += 1;
            const int k0 = max(0, L - 5), k1 = min(L, 32);
            for (int k = k0; k < k1; ++k) acc[k] += (u32)(e >> k) + 1u + (u32)k;
        }
        __syncwarp();
        for (int L = lane; L < 66; L += 32) {
            u32 h = 0;
            for (int j = 0; j < 32; ++j) h += sh.hl[wi][j][L];
            sh.hs[wi][L] = h;
        }
        __syncwarp();
        // lane = k: the exact terms of all lanes, then the histogram terms
        {
            const int k = lane;
            u32 s = 0, le = 0, gt = 0;  // exact terms, escapes with L <= k, escapes with L > k + 5
            for (int j = 0; j < 32; ++j) s += sh.acc[wi][j][k];
            for (int L = 0; L < 66; ++L) {
                const u32 h = sh.hs[wi][L];
                if (L <= k) le += h;
                else if (L > k + 5) gt += h;
            }
            sh.cost[wi][w][k] = cnt * (u32)w + s + le * (1u + (u32)k) + gt * (97u + (u32)k);
        }
        __syncwarp();
    }
    // argmin over (w, k): lane k scans w, then a warp argmin (ties: smallest w, then k)
    u32 best = 0xffffffffu, bw = 0;
    for (int w = 0; w <= 32; ++w) {
        const u32 c = sh.cost[wi][w][lane];
        if (c < best) {
            best = c;
            bw = (u32)w;
        }
    }
    u64 key = ((u64)best << 32) | (bw << 8) | (u32)lane;
    for (int d = 16; d > 0; d >>= 1) {
        const u64 o = __shfl_xor_sync(kFullMask, key, d);
        key = o < key ? o : key;
    }
    if (lane == 0) {
        wout[b] = (u8)((key >> 8) & 0xffu);
        kout[b] = (u8)(key & 0xffu);
        if (cost_out) cost_out[b] = (u32)(key >> 32);
    }
}

// ------------------------------------------------------------------ cost ----------------
__device__ __forceinline__ u32 warp_block_cost(const u64* p, u32 cnt, int w, int k, int lane) {
    const u64 thr = escape_threshold(w);
    u32 s = 0;
    for (u32 i = lane; i < cnt; i += 32) {
        const u64 x = p[i];
        s += (u32)w + (x >= thr ? esc_len(x - thr, k) : 0u);
    }
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(kFullMask, s, d);
    return s;
}

__global__ void __launch_bounds__(32 * WARPS) cost_kernel(const u64* __restrict__ v, u64 n, u64 nblk,
                                                          const u8* __restrict__ win, const u8* __restrict__ kin,
                                                          u32* __restrict__ cost) {
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b = (u64)blockIdx.x * WARPS + wi;
    if (b >= nblk) return;
    const u32 c = warp_block_cost(v + b * BLK, block_count(n, b), min((int)win[b], 32), min((int)kin[b], 31), lane);
    if (lane == 0) cost[b] = c;
}

// ------------------------------------------------------------ encode / decode -----------
__device__ __forceinline__ void or_bits(u32* words, u64 pos, u64 val, u32 nbits) {
    // LSB-first: val's low nbits at bit pos (nbits <= 64)
    if (!nbits) return;
    const u64 wk = pos >> 5;
    const u32 o = (u32)(pos & 31u);
    const u64 lo = nbits < 64 ? (val & ((1ull << nbits) - 1ull)) : val;
    atomicOr(&words[wk], (u32)(lo << o));
    if (o + nbits > 32) atomicOr(&words[wk + 1], (u32)(lo >> (32 - o)));
    if (o + nbits > 64) atomicOr(&words[wk + 2], (u32)((lo >> (32 - o)) >> 32));
}

// warp exclusive prefix sum; *total receives the sum over the warp
__device__ __forceinline__ u32 warp_excl(u32 v, u32* total) {
    const int lane = threadIdx.x & 31;
    u32 incl = v;
    for (int d = 1; d < 32; d <<= 1) {
        const u32 o = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += o;
    }
    *total = __shfl_sync(kFullMask, incl, 31);
    return incl - v;
}

// Encoder: block offsets (exclusive prefix of the costs, bits) are given.  The payload must
// be zeroed.
__global__ void __launch_bounds__(32 * WARPS) encode_kernel(const u64* __restrict__ v, u64 n, u64 nblk,
                                                            const u8* __restrict__ win, const u8* __restrict__ kin,
                                                            const u64* __restrict__ offs, u32* __restrict__ payload) {
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b = (u64)blockIdx.x * WARPS + wi;
    if (b >= nblk) return;
    const u32 cnt = block_count(n, b);
    const int w = min((int)win[b], 32), k = min((int)kin[b], 31);
    const u64 thr = escape_threshold(w);
    const u64* p = v + b * BLK;
    // pass 1: sizes of the U region and escape counts
    u32 ubits = 0, nesc = 0;
    for (u32 i = lane; i < cnt; i += 32) {
        const u64 x = p[i];
        if (x >= thr) {
            const u64 q = (x - thr) >> k;
            ubits += (u32)min(q, (u64)32) + 1u;
            ++nesc;
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        ubits += __shfl_xor_sync(kFullMask, ubits, d);
        nesc += __shfl_xor_sync(kFullMask, nesc, d);
    }
    const u64 s0 = offs[b], u0 = s0 + (u64)cnt * (u64)w, r0 = u0 + ubits, x0 = r0 + (u64)nesc * (u64)k;
    // pass 2: write the regions
    u64 upos = u0;
    u32 erank = 0, crank = 0;
    for (u32 i0 = 0; i0 < cnt; i0 += 32) {
        const u32 i = i0 + lane;
        const bool ok = i < cnt;
        const u64 x = ok ? p[i] : 0ull;
        const bool esc = ok && x >= thr;
        if (ok) or_bits(payload, s0 + (u64)i * (u64)w, esc ? thr : x, (u32)w);
        const u64 e = esc ? x - thr : 0ull;
        const u64 q = e >> k;
        const bool capped = esc && q >= 32;
        const u32 ulen = esc ? (u32)min(q, (u64)32) + 1u : 0u;
        u32 utot, etot, ctot;
        const u32 uoff = warp_excl(ulen, &utot);
        const u32 eoff = warp_excl(esc ? 1u : 0u, &etot);
        const u32 coff = warp_excl(capped ? 1u : 0u, &ctot);
        if (esc) {
            or_bits(payload, upos + uoff, (1ull << (ulen - 1)) - 1ull, ulen);  // ulen-1 ones, a zero
            or_bits(payload, r0 + (u64)(erank + eoff) * (u64)k, e, (u32)k);
            if (capped) or_bits(payload, x0 + (u64)(crank + coff) * 64ull, e, 64u);
        }
        upos += utot;
        erank += etot;
        crank += ctot;
    }
}

// Decoder: one warp per block.  Lanes read the slots, locate the zeros of the U region by a
// warp scan of its words, then read each escape's remainder and capped value.
__global__ void __launch_bounds__(32 * WARPS) decode_kernel(const u32* __restrict__ payload, u64 payload_bits, u64 n,
                                                            u64 nblk, const u8* __restrict__ win,
                                                            const u8* __restrict__ kin, const u64* __restrict__ offs,
                                                            u64* __restrict__ out, u32* err) {
    __shared__ u32 szero[WARPS][BLK];  // position of the j-th zero of U, relative to U's start
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const u64 b = (u64)blockIdx.x * WARPS + wi;
    if (b >= nblk) return;
    const u32 cnt = block_count(n, b);
    const int w = win[b], k = kin[b];
    const u64 base = offs[b];
    if (w > 32 || k > 31 || base > payload_bits || (u64)cnt * (u64)w > payload_bits - base) {
        if (lane == 0) atomicOr(err, kErrBadStream);
        return;
    }
    const u64 thr = escape_threshold(w);
    const u64 nwords = (payload_bits + 31) >> 5;
    auto word = [&](u64 i) -> u32 { return i < nwords ? __ldg(&payload[i]) : 0u; };
    auto peek64 = [&](u64 pos) -> u64 {
        const u64 i = pos >> 5;
        const u32 o = (u32)(pos & 31u);
        const u64 lo = (u64)word(i) | ((u64)word(i + 1) << 32);
        return o ? ((lo >> o) | ((u64)word(i + 2) << (64 - o))) : lo;
    };
    // slots
    u32 esc_mask[PER_LANE];
    u32 nesc = 0;
    u64 xs[PER_LANE];
#pragma unroll
    for (int r = 0; r < PER_LANE; ++r) {
        const u32 i = (u32)r * 32 + lane;
        u64 s = 0;
        if (i < cnt && w) s = peek64(base + (u64)i * (u64)w) & thr;
        const bool esc = i < cnt && s == thr;
        xs[r] = s;
        esc_mask[r] = __ballot_sync(kFullMask, esc);
        nesc += __popc(esc_mask[r]);
    }
    const u64 u0 = base + (u64)cnt * (u64)w;
    // zeros of U: 32-bit chunks (lane j: bits u0 + 32 * (32 c + j) ...), until nesc found
    u32 found = 0;
    for (u64 c0 = 0; found < nesc; c0 += 32 * 32) {
        const u64 pos = u0 + c0 + 32ull * lane;
        const u32 bits = pos < payload_bits ? (u32)peek64(pos) : 0u;
        u32 zeros = ~bits;
        if (pos + 32 > payload_bits) zeros &= pos >= payload_bits ? 0u : ((1u << (payload_bits - pos)) - 1u);
        u32 ztot;
        const u32 zoff = warp_excl((u32)__popc(zeros), &ztot);
        u32 j = found + zoff;
        while (zeros && j < nesc) {
            const int bpos = __ffs((int)zeros) - 1;
            zeros &= zeros - 1;
            szero[wi][j++] = (u32)(c0 + 32ull * lane + (u64)bpos);
        }
        found += ztot;
        if (c0 > 33ull * BLK + 64) break;  // more bits than any block's U region: corrupt
    }
    __syncwarp();
    if (found < nesc) {
        if (lane == 0) atomicOr(err, kErrBadStream);
        return;
    }
    const u64 r0 = nesc ? u0 + szero[wi][nesc - 1] + 1 : u0;
    const u64 x0 = r0 + (u64)nesc * (u64)k;
    u32 before = 0, cbefore = 0;
#pragma unroll
    for (int r = 0; r < PER_LANE; ++r) {
        const u32 i = (u32)r * 32 + lane;
        const u32 m = esc_mask[r];
        const bool esc = (m >> lane) & 1u;
        u64 x = xs[r];
        u32 q = 0;
        if (esc) {
            const u32 j = before + __popc(m & ((1u << lane) - 1u));
            const u32 zj = szero[wi][j], zp = j ? szero[wi][j - 1] + 1 : 0u;
            q = zj - zp;
            const u64 rem = k ? (peek64(r0 + (u64)j * (u64)k) & ((1ull << k) - 1ull)) : 0ull;
            x = thr + (((u64)q << k) | rem);
        }
        const bool capped = esc && q >= 32;
        const u32 cm = __ballot_sync(kFullMask, capped);
        if (capped) x = thr + peek64(x0 + 64ull * (cbefore + __popc(cm & ((1u << lane) - 1u))));
        if (i < cnt) out[b * BLK + i] = x;
        before += __popc(m);
        cbefore += __popc(cm);
    }
    if (lane == 0 && x0 + 64ull * cbefore > payload_bits) atomicOr(err, kErrBadStream);
}

// Exclusive prefix sum of the block costs (bits) -> offsets, single CTA (block counts are
// ~n / 1024).  total receives the payload size in bits.
__global__ void __launch_bounds__(1024) offsets_kernel(const u32* __restrict__ cost, u64 nblk, u64* __restrict__ offs,
                                                       u64* total) {
    __shared__ u64 scratch[40];
    u64 carry = 0;
    for (u64 s = 0; s < nblk; s += 1024) {
        const u64 i = s + threadIdx.x;
        const u64 c = i < nblk ? cost[i] : 0ull;
        u64 tot;
        const u64 ex = block_exclusive<1024>(c, 0ull, AddOp{}, scratch, tot);
        if (i < nblk) offs[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0) *total = carry;
}

// Learned mode: blocks whose weaker head has confidence at or below thr get the exhaustive
// search (thr = 0: none, thr = 1: all).
__global__ void fallback_kernel(const float* __restrict__ conf, u64 nblk, float thr, u8* __restrict__ flags,
                                unsigned long long* count) {
    u32 c = 0;
    for (u64 b = (u64)blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += (u64)gridDim.x * blockDim.x) {
        const bool f = fminf(conf[2 * b], conf[2 * b + 1]) <= thr;
        flags[b] = f ? 1 : 0;
        c += f;
    }
    for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(kFullMask, c, d);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

__global__ void sum_kernel(const u64* __restrict__ v, u64 n, double* sum) {
    double s = 0.0;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        s += (double)v[i];
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(kFullMask, s, d);
    if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(sum, s);
}

// One parameter pair for the whole stream, chosen the way the plain method chooses its
// Golomb-Rice parameter (floor(log2(mean)), 0 below a mean of 1): w = 0, k = that (<= 31).
__global__ void fill_global_kernel(const double* sum, u64 n, u64 nblk, u8* __restrict__ w, u8* __restrict__ k) {
    const double mean = n ? *sum / (double)n : 0.0;
    int kk = 0;
    if (mean >= 1.0) {
        const u64 m = mean >= 1.8e19 ? ~0ull : (u64)mean;
        kk = (int)bitlen64(m) - 1;
    }
    kk = min(kk, 31);
    for (u64 b = (u64)blockIdx.x * blockDim.x + threadIdx.x; b < nblk; b += (u64)gridDim.x * blockDim.x) {
        w[b] = 0;
        k[b] = (u8)kk;
    }
}

inline unsigned grid_for(u64 nblk) { return (unsigned)((nblk + WARPS - 1) / WARPS); }
inline unsigned grid_flat(u64 n) {
    u64 g = (n + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    return (unsigned)(g ? g : 1);
}

}  // namespace

void launch_block_features(const unsigned long long* v, uint64_t n, float* feats, cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (nblk) features_kernel<<<grid_for(nblk), 32 * WARPS, 0, st>>>(v, n, nblk, feats);
}
void launch_block_search(const unsigned long long* v, uint64_t n, const uint8_t* only, uint8_t* w, uint8_t* k,
                         uint32_t* cost, cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (!nblk) return;
    const int smem = (int)sizeof(SearchShared);
    cudaFuncSetAttribute(search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    search_kernel<<<grid_for(nblk), 32 * WARPS, smem, st>>>(v, n, nblk, only, w, k, cost);
}
void launch_block_cost(const unsigned long long* v, uint64_t n, const uint8_t* w, const uint8_t* k, uint32_t* cost,
                       cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (nblk) cost_kernel<<<grid_for(nblk), 32 * WARPS, 0, st>>>(v, n, nblk, w, k, cost);
}
void launch_block_offsets(const uint32_t* cost, uint64_t nblk, unsigned long long* offs, unsigned long long* total,
                          cudaStream_t st) {
    offsets_kernel<<<1, 1024, 0, st>>>(cost, nblk, offs, total);
}
void launch_block_encode(const unsigned long long* v, uint64_t n, const uint8_t* w, const uint8_t* k,
                         const unsigned long long* offs, uint32_t* payload, cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (nblk) encode_kernel<<<grid_for(nblk), 32 * WARPS, 0, st>>>(v, n, nblk, w, k, offs, payload);
}
void launch_block_fallback(const float* conf, uint64_t nblk, float thr, uint8_t* flags, unsigned long long* count,
                           cudaStream_t st) {
    if (nblk) fallback_kernel<<<grid_flat(nblk), 256, 0, st>>>(conf, nblk, thr, flags, count);
}
void launch_block_global(const unsigned long long* v, uint64_t n, double* sum, uint8_t* w, uint8_t* k,
                         cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (!nblk) return;
    sum_kernel<<<grid_flat(n), 256, 0, st>>>(v, n, sum);
    fill_global_kernel<<<grid_flat(nblk), 256, 0, st>>>(sum, n, nblk, w, k);
}
void launch_block_decode(const uint32_t* payload, uint64_t payload_bits, uint64_t n, const uint8_t* w,
                         const uint8_t* k, const unsigned long long* offs, unsigned long long* out, uint32_t* err,
                         cudaStream_t st) {
    const u64 nblk = (n + BLK - 1) / BLK;
    if (nblk)
        decode_kernel<<<grid_for(nblk), 32 * WARPS, 0, st>>>(payload, payload_bits, n, nblk, w, k, offs, out, err);
}

}  // namespace dev
}  // namespace xnyz
