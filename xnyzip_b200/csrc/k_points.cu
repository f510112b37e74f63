// Point-level kernels: bounding-box minimum (shift_points), quantization with range and
// error statistics, and sort-key generation for block and direct mode.
//
// Reference behaviour restated here (paths relative to the reference's source/):
//   shift_points           preprocessor/shifting.hpp:11-36  (strict '<' scan from FLT_MAX)
//   quantize               quantizer/truncated_octahedron_quantizer.hpp:21-55, cube_quantizer.hpp:15-27,
//                          adaptive_quantizer.hpp:16-81
//   ranges / direct switch composer/block_compressor.hpp:69-88
//   error statistics       composer/block_compressor_rle.hpp:53-67
//   block keys             quantizer/block_quantizer.hpp:93-115
//   direct keys            composer/block_compressor.hpp:90-101
#include <cfloat>

#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int kThreads = 256;

// Grid-stride loop over points that issues the loads of U points (U strides apart) before
// processing them, so that each thread keeps U loads in flight.  body(i, x, y, z).
template <int U, typename F>
__device__ __forceinline__ void for_each_point(const float* __restrict__ xyz, u64 n, F&& body) {
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 i0 = (u64)blockIdx.x * kThreads + threadIdx.x; i0 < n; i0 += U * stride) {
        float x[U], y[U], z[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const u64 i = i0 + (u64)u * stride;
            if (i < n) {
                x[u] = __ldg(xyz + 3 * i);
                y[u] = __ldg(xyz + 3 * i + 1);
                z[u] = __ldg(xyz + 3 * i + 2);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const u64 i = i0 + (u64)u * stride;
            if (i < n) body(i, x[u], y[u], z[u]);
        }
    }
}

// Order key of a float for the minimum scan: monotone in value, +0 and -0 equal, NaN last.
__device__ __forceinline__ u32 order_key(float f) {
    u32 b = __float_as_uint(f);
    if ((b & 0x7fffffffu) > 0x7f800000u) return 0xffffffffu;  // NaN never wins ('<' is false)
    if ((b & 0x7fffffffu) == 0u) b = 0u;                        // -0 ties with +0
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) { return a < b ? a : b; }

// Minimum over the block of three u64 values, then one atomicMin per axis.
__device__ void block_min3(unsigned long long m[3], unsigned long long* dst) {
    __shared__ unsigned long long sm[3][kThreads / 32];
    for (int a = 0; a < 3; ++a) {
        unsigned long long v = m[a];
        for (int d = 16; d > 0; d >>= 1) v = umin64(v, __shfl_xor_sync(kFullMask, v, d));
        if (lane_id() == 0) sm[a][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        unsigned long long v = sm[threadIdx.x][0];
        for (int w = 1; w < kThreads / 32; ++w) v = umin64(v, sm[threadIdx.x][w]);
        atomicMin(&dst[threadIdx.x], v);
    }
}

// Maximum over the block of three u32 order keys, then one atomicMax per axis.
__device__ void block_max3(u32 m[3], unsigned int* dst) {
    __shared__ u32 sm[3][kThreads / 32];
    for (int a = 0; a < 3; ++a) {
        u32 v = m[a];
        for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(kFullMask, v, d));
        if (lane_id() == 0) sm[a][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        u32 v = sm[threadIdx.x][0];
        for (int w = 1; w < kThreads / 32; ++w) v = max(v, sm[threadIdx.x][w]);
        atomicMax(&dst[threadIdx.x], v);
    }
}

// shift_points keeps the first of equal minima; the key packs (order key, index) so the
// smallest index wins ties (including +0 / -0), and the initial FLT_MAX candidate carries
// index 0xffffffff.  The largest order key per axis feeds the adaptive quantizer's steps.
__global__ void __launch_bounds__(kThreads) bbox_kernel(const float* __restrict__ xyz, u64 n, PointStats* stats) {
    unsigned long long m[3];
    u32 mx[3];
    for (int a = 0; a < 3; ++a) {
        m[a] = ~0ull;
        mx[a] = 0u;
    }
    for_each_point<4>(xyz, n, [&](u64 i, float x, float y, float z) {
        const float v[3] = {x, y, z};
        for (int a = 0; a < 3; ++a) {
            const u32 ok = order_key(v[a]);
            m[a] = umin64(m[a], ((unsigned long long)ok << 32) | (u32)i);
            mx[a] = max(mx[a], ok);
        }
    });
    block_min3(m, stats->minkey);
    block_max3(mx, stats->maxkey);
}

__device__ __forceinline__ float order_key_value(u32 k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

__device__ __forceinline__ void load_offset(const float* xyz, const PointStats* st, float off[3]) {
    for (int a = 0; a < 3; ++a) {
        const unsigned long long k = st->minkey[a];
        const u32 idx = (u32)(k & 0xffffffffu);
        const u32 ok = (u32)(k >> 32);
        // The reference starts from FLT_MAX; a candidate wins only if strictly smaller.
        off[a] = (idx == 0xffffffffu || ok >= order_key(FLT_MAX)) ? FLT_MAX : xyz[3 * (u64)idx + a];
    }
}

__device__ __forceinline__ bool finite3(float x, float y, float z) {
    return isfinite(x) && isfinite(y) && isfinite(z);
}

// AdaptiveQuantizer::quantize's steps (quantizer/adaptive_quantizer.hpp:42-64).  Over the
// shifted points the minimum is 0 (the offset is the minimum) and the maximum is
// max - offset (float subtraction is monotone), each compared against the scan's start
// values (FLT_MAX, and the smallest normal float for the maxima).  One thread, IEEE
// single-precision operations in the reference's order.
__global__ void adaptive_steps_kernel(const float* __restrict__ xyz, float R, PointStats* stats) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float off[3];
    load_offset(xyz, stats, off);
    float d[3];
    for (int a = 0; a < 3; ++a) {
        const float hi = __fsub_rn(order_key_value(stats->maxkey[a]), off[a]);
        const float mx = (FLT_MIN < hi) ? hi : FLT_MIN;
        const float lo = __fsub_rn(off[a], off[a]);  // the minimum's own shifted value
        const float mn = (lo < FLT_MAX) ? lo : FLT_MAX;
        d[a] = __fsub_rn(mx, mn);
    }
    const float norm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])),
                                            __fmul_rn(d[2], d[2])));
    for (int a = 0; a < 3; ++a)
        stats->step[a] = norm > 0.0f ? __fdiv_rn(__fmul_rn(R, d[a]), norm) : __fdiv_rn(R, __fsqrt_rn(3.0f));
}

__global__ void __launch_bounds__(kThreads) quantize_range_kernel(const float* __restrict__ xyz, u64 n,
                                                                  QuantParams q, PointStats* stats,
                                                                  int with_error_stats, i32* __restrict__ cells) {
    __shared__ float off[3];
    __shared__ int smax[3][kThreads / 32], smin[3][kThreads / 32];
    __shared__ u32 snf[kThreads / 32], smse[kThreads / 32];
    __shared__ double ssum[kThreads / 32];
    if (threadIdx.x == 0) {
        load_offset(xyz, stats, off);
        if (blockIdx.x == 0)
            for (int a = 0; a < 3; ++a) stats->offset[a] = off[a];
    }
    __syncthreads();
    const float ox = off[0], oy = off[1], oz = off[2];
    int mx[3] = {0, 0, 0};
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX};
    u32 nonfinite = 0;
    float emax = 0.0f;
    double esum = 0.0;
    for_each_point<4>(xyz, n, [&](u64 i, float x, float y, float z) {
        if (!finite3(x, y, z)) {
            ++nonfinite;
            return;
        }
        const float px = __fsub_rn(x, ox), py = __fsub_rn(y, oy), pz = __fsub_rn(z, oz);
        i32 c[3];
        quantize(q, px, py, pz, c[0], c[1], c[2]);
        if (cells) {  // kept for the key kernel (keys_cells_kernel), which then need not quantize again
            cells[3 * i] = c[0];
            cells[3 * i + 1] = c[1];
            cells[3 * i + 2] = c[2];
        }
        for (int a = 0; a < 3; ++a) {
            mx[a] = max(mx[a], c[a]);
            mn[a] = min(mn[a], c[a]);
        }
        if (with_error_stats) {
            // (sx - rx)^2 + (sy - ry)^2 + (sz - rz)^2 in float, left to right.
            float rx, ry, rz;
            recover(q, c[0], c[1], c[2], 0.0f, 0.0f, 0.0f, rx, ry, rz);
            const float dx = __fsub_rn(px, rx), dy = __fsub_rn(py, ry), dz = __fsub_rn(pz, rz);
            const float e = __fadd_rn(__fadd_rn(sqf(dx), sqf(dy)), sqf(dz));
            emax = fmaxf(emax, e);
            esum += (double)e;
        }
    });
    for (int d = 16; d > 0; d >>= 1) {
        for (int a = 0; a < 3; ++a) {
            mx[a] = max(mx[a], __shfl_xor_sync(kFullMask, mx[a], d));
            mn[a] = min(mn[a], __shfl_xor_sync(kFullMask, mn[a], d));
        }
        nonfinite += __shfl_xor_sync(kFullMask, nonfinite, d);
        emax = fmaxf(emax, __shfl_xor_sync(kFullMask, emax, d));
        esum += __shfl_xor_sync(kFullMask, esum, d);
    }
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0) {
        for (int a = 0; a < 3; ++a) {
            smax[a][w] = mx[a];
            smin[a][w] = mn[a];
        }
        snf[w] = nonfinite;
        smse[w] = __float_as_uint(emax);
        ssum[w] = esum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int bx[3] = {0, 0, 0}, bn[3] = {INT_MAX, INT_MAX, INT_MAX};
        u32 nf = 0, em = 0;
        double es = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            for (int a = 0; a < 3; ++a) {
                bx[a] = max(bx[a], smax[a][k]);
                bn[a] = min(bn[a], smin[a][k]);
            }
            nf += snf[k];
            em = max(em, smse[k]);
            es += ssum[k];
        }
        for (int a = 0; a < 3; ++a) {
            atomicMax(&stats->max_cell[a], bx[a]);
            atomicMin(&stats->min_cell[a], bn[a]);
        }
        if (nf) atomicAdd(&stats->nonfinite, nf);
        if (with_error_stats) {
            atomicMax(&stats->mse_max_bits, em);
            atomicAdd(&stats->mse_sum, es);
        }
    }
}

// Per-block histograms of the sort digits, flushed with one atomicAdd per non-zero bin.
struct DigitHist {
    u32* s;  // shared [passes * 256]
    int passes;
    __device__ __forceinline__ void add(u64 key) {
        for (int p = 0; p < passes; ++p) atomicAdd(&s[p * 256 + (u32)((key >> (8 * p)) & 255u)], 1u);
    }
};

__device__ __forceinline__ void stage_hilbert_table(const u8* g, u8* s) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) s[i] = g ? g[i] : 0;
}

// Block mode: key = id << 21 | quad << 18 | sfc18 with the reference's size_t arithmetic
// (negative lattice indices wrap to 2^64 + v before the division by 64).
__device__ __forceinline__ u64 block_key(i32 x, i32 y, i32 z, const BlockKeyParams& kp, const u8* htab) {
    const u64 X = (u64)(i64)x, Y = (u64)(i64)y, Z = (u64)(i64)z;
    const u64 cx = X >> 6, cy = Y >> 6, cz = Z >> 6;
    const u32 dx = (u32)(X & 63u), dy = (u32)(Y & 63u), dz = (u32)(Z & 63u);
    const u64 m = kp.hilbert ? (u64)hilbert_code6(htab, dx, dy, dz, kp.hstart) : morton3((i32)dx, (i32)dy, (i32)dz);
    const u64 quad = (cx & 1u) | ((cy & 1u) << 1) | ((cz & 1u) << 2);
    const u64 low = (quad << 18) | m;
    const u64 xy = (cx >> 1) + (cy >> 1) * kp.nx;
    if (z >= 0) return ((xy + (cz >> 1) * kp.nx * kp.ny) << 21) | low;
    return kp.defect_flag | (xy << 21) | low;  // z == -1: id = xy + defect_base
}

__global__ void __launch_bounds__(kThreads) keys_block_kernel(const float* __restrict__ xyz, u64 n, QuantParams q,
                                                              const PointStats* stats, BlockKeyParams kp,
                                                              const u8* __restrict__ htab_g,
                                                              unsigned long long* __restrict__ keys,
                                                              u32* __restrict__ payload, int passes, u32* hist) {
    __shared__ float off[3];
    __shared__ u8 htab[256];
    __shared__ u32 sh[8 * 256];
    if (threadIdx.x == 0) load_offset(xyz, stats, off);
    stage_hilbert_table(htab_g, htab);
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) sh[i] = 0;
    __syncthreads();
    DigitHist dh{sh, passes};
    for_each_point<4>(xyz, n, [&](u64 i, float fx, float fy, float fz) {
        const float px = __fsub_rn(fx, off[0]), py = __fsub_rn(fy, off[1]), pz = __fsub_rn(fz, off[2]);
        i32 x, y, z;
        quantize(q, px, py, pz, x, y, z);
        const u64 k = block_key(x, y, z, kp, htab);
        keys[i] = k;
        if (payload) payload[i] = (u32)i;
        if (passes) dh.add(k);
    });
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Cell tables (encode_cells_with_counts, composer/block_compressor_rle.hpp:341-470): block
// keys straight from int32 lattice cells, and the per-axis minima / maxima of the cells.
__global__ void __launch_bounds__(kThreads) keys_cells_kernel(const i32* __restrict__ cells, u64 n, BlockKeyParams kp,
                                                              const u8* __restrict__ htab_g,
                                                              unsigned long long* __restrict__ keys,
                                                              u32* __restrict__ payload, int passes, u32* hist) {
    __shared__ u8 htab[256];
    __shared__ u32 sh[8 * 256];
    stage_hilbert_table(htab_g, htab);
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) sh[i] = 0;
    __syncthreads();
    DigitHist dh{sh, passes};
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        const u64 k = block_key(__ldg(cells + 3 * i), __ldg(cells + 3 * i + 1), __ldg(cells + 3 * i + 2), kp, htab);
        keys[i] = k;
        if (payload) payload[i] = (u32)i;
        if (passes) dh.add(k);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__global__ void __launch_bounds__(kThreads) cells_stats_kernel(const i32* __restrict__ cells, u64 n,
                                                               PointStats* stats) {
    i32 lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride)
        for (int a = 0; a < 3; ++a) {
            const i32 v = __ldg(cells + 3 * i + a);
            lo[a] = min(lo[a], v);
            hi[a] = max(hi[a], v);
        }
    for (int a = 0; a < 3; ++a) {
        for (int d = 16; d > 0; d >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(kFullMask, lo[a], d));
            hi[a] = max(hi[a], __shfl_xor_sync(kFullMask, hi[a], d));
        }
        if (lane_id() == 0) {
            atomicMin(&stats->min_cell[a], lo[a]);
            atomicMax(&stats->max_cell[a], hi[a]);
        }
    }
}

__global__ void gather_i32_kernel(const i32* __restrict__ src, const u32* __restrict__ idx, u64 n,
                                  i32* __restrict__ dst) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

// expand_cells_to_points (composer/block_decompressor_rle.hpp:339-358): every cell repeated
// counts[i] times, recovered and unshifted; output positions by a chained scan of the counts.
__global__ void __launch_bounds__(kThreads) expand_cells_kernel(const i32* __restrict__ cells,
                                                                const i32* __restrict__ counts, u64 n, QuantParams q,
                                                                const float* __restrict__ off3, LookBackState lb,
                                                                u32* tile_counter, float* __restrict__ out, u64 cap,
                                                                unsigned long long* total, u32* err) {
    constexpr int kItems = 16, kTile = kThreads * kItems;
    __shared__ u64 scratch[16];
    __shared__ u32 slot;
    __shared__ u64 sbase;
    const u32 tile = claim_tile(tile_counter, &slot);
    const u64 base = (u64)tile * kTile + (u64)threadIdx.x * kItems;
    u64 s = 0;
    for (int i = 0; i < kItems; ++i)
        if (base + i < n) s += (u64)max(__ldg(counts + base + i), 0);
    u64 tot;
    const u64 ex = block_exclusive<kThreads>(s, 0ull, AddOp{}, scratch, tot);
    if (threadIdx.x < 32) {
        LookBack64 l{lb.flag, lb.agg, lb.inc};
        const u64 r = warp_lookback_add(l, tile, tot, err);
        if (threadIdx.x == 0) {
            sbase = r;
            if (tile == gridDim.x - 1) *total = r + tot;
        }
    }
    __syncthreads();
    u64 pos = sbase + ex;
    const float ox = off3[0], oy = off3[1], oz = off3[2];
    for (int i = 0; i < kItems; ++i) {
        const u64 j = base + i;
        if (j >= n) break;
        const u64 c = (u64)max(__ldg(counts + j), 0);
        if (pos + c > cap) {
            atomicOr(err, kErrOverflow);
            break;
        }
        float x, y, z;
        recover(q, __ldg(cells + 3 * j), __ldg(cells + 3 * j + 1), __ldg(cells + 3 * j + 2), ox, oy, oz, x, y, z);
        for (u64 r = 0; r < c; ++r) {
            out[3 * (pos + r)] = x;
            out[3 * (pos + r) + 1] = y;
            out[3 * (pos + r) + 2] = z;
        }
        pos += c;
    }
}

// Direct mode: key = global Morton or Hilbert code (hilbert_bits levels); z == -1 cells keep
// their transformed low levels under defect_flag.
__global__ void __launch_bounds__(kThreads) keys_direct_kernel(const float* __restrict__ xyz, u64 n, QuantParams q,
                                                               const PointStats* stats, DirectKeyParams kp,
                                                               const u8* __restrict__ htab_g,
                                                               unsigned long long* __restrict__ keys,
                                                               u32* __restrict__ payload, int passes, u32* hist) {
    __shared__ float off[3];
    __shared__ u8 htab[256];
    __shared__ u32 sh[8 * 256];
    if (threadIdx.x == 0) load_offset(xyz, stats, off);
    stage_hilbert_table(htab_g, htab);
    for (int i = threadIdx.x; i < passes * 256; i += kThreads) sh[i] = 0;
    __syncthreads();
    DigitHist dh{sh, passes};
    for_each_point<4>(xyz, n, [&](u64 i, float fx, float fy, float fz) {
        const float px = __fsub_rn(fx, off[0]), py = __fsub_rn(fy, off[1]), pz = __fsub_rn(fz, off[2]);
        i32 x, y, z;
        quantize(q, px, py, pz, x, y, z);
        u64 m = morton3(x, y, z);
        if (kp.hilbert) m = hilbert_apply(htab, m, kp.bits, 0u);
        const u64 k = (z >= 0) ? m : (kp.defect_flag | (m & (kp.defect_flag - 1)));
        keys[i] = k;
        if (payload) payload[i] = (u32)i;
        if (passes) dh.add(k);
    });
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

__global__ void __launch_bounds__(kThreads) quantize_cells_kernel(const float* __restrict__ xyz, u64 n, QuantParams q,
                                                                  const PointStats* stats, i32* __restrict__ cells) {
    __shared__ float off[3];
    if (threadIdx.x == 0) load_offset(xyz, stats, off);
    __syncthreads();
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        const float px = __fsub_rn(xyz[3 * i], off[0]);
        const float py = __fsub_rn(xyz[3 * i + 1], off[1]);
        const float pz = __fsub_rn(xyz[3 * i + 2], off[2]);
        quantize(q, px, py, pz, cells[3 * i], cells[3 * i + 1], cells[3 * i + 2]);
    }
}

__global__ void __launch_bounds__(kThreads) recover_cells_kernel(const i32* __restrict__ cells, u64 n, QuantParams q,
                                                                 const float* __restrict__ off,
                                                                 float* __restrict__ xyz) {
    const u64 stride = (u64)gridDim.x * kThreads;
    const float ox = off[0], oy = off[1], oz = off[2];
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
        float x, y, z;
        recover(q, cells[3 * i], cells[3 * i + 1], cells[3 * i + 2], ox, oy, oz, x, y, z);
        xyz[3 * i] = x;
        xyz[3 * i + 1] = y;
        xyz[3 * i + 2] = z;
    }
}

__global__ void __launch_bounds__(kThreads) hilbert_kernel(const unsigned long long* __restrict__ in, u64 n,
                                                           const u8* __restrict__ tab_g, int top, u32 state,
                                                           unsigned long long* __restrict__ out) {
    __shared__ u8 tab[256];
    stage_hilbert_table(tab_g, tab);
    __syncthreads();
    const u64 stride = (u64)gridDim.x * kThreads;
    for (u64 i = (u64)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) out[i] = hilbert_apply(tab, in[i], top, state);
}

int grid_for(u64 n) {
    // Persistent-style grid: a few resident blocks per SM of the 148-SM B200.
    u64 want = (n + kThreads - 1) / kThreads;
    u64 cap = 148ull * 8ull;
    if (want < 1) want = 1;
    return (int)(want < cap ? want : cap);
}

}  // namespace

void launch_bbox(const float* xyz, uint64_t n, PointStats* stats, cudaStream_t st) {
    bbox_kernel<<<grid_for(n), kThreads, 0, st>>>(xyz, n, stats);
}
void launch_adaptive_steps(const float* xyz, float l2, PointStats* stats, cudaStream_t st) {
    adaptive_steps_kernel<<<1, 32, 0, st>>>(xyz, l2, stats);
}
void launch_quantize_range(const float* xyz, uint64_t n, QuantParams q, PointStats* stats, int with_error_stats,
                           cudaStream_t st, int32_t* cells) {
    quantize_range_kernel<<<grid_for(n), kThreads, 0, st>>>(xyz, n, q, stats, with_error_stats, cells);
}
void launch_keys_block(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, BlockKeyParams kp,
                       const uint8_t* hilbert_tab, unsigned long long* keys, uint32_t* payload, int passes,
                       uint32_t* hist, cudaStream_t st) {
    keys_block_kernel<<<grid_for(n), kThreads, 0, st>>>(xyz, n, q, stats, kp, hilbert_tab, keys, payload, passes,
                                                        hist);
}
void launch_keys_direct(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, DirectKeyParams kp,
                        const uint8_t* hilbert_tab, unsigned long long* keys, uint32_t* payload, int passes,
                        uint32_t* hist, cudaStream_t st) {
    keys_direct_kernel<<<grid_for(n), kThreads, 0, st>>>(xyz, n, q, stats, kp, hilbert_tab, keys, payload, passes,
                                                         hist);
}
void launch_keys_cells(const int32_t* cells, uint64_t n, BlockKeyParams kp, const uint8_t* hilbert_tab,
                       unsigned long long* keys, uint32_t* payload, int passes, uint32_t* hist, cudaStream_t st) {
    keys_cells_kernel<<<grid_for(n), kThreads, 0, st>>>(cells, n, kp, hilbert_tab, keys, payload, passes, hist);
}
void launch_cells_stats(const int32_t* cells, uint64_t n, PointStats* stats, cudaStream_t st) {
    cells_stats_kernel<<<grid_for(n), kThreads, 0, st>>>(cells, n, stats);
}
void launch_gather_i32(const int32_t* src, const uint32_t* idx, uint64_t n, int32_t* dst, cudaStream_t st) {
    if (n) gather_i32_kernel<<<grid_for(n), kThreads, 0, st>>>(src, idx, n, dst);
}
void launch_expand_cells(const int32_t* cells, const int32_t* counts, uint64_t n, QuantParams q, const float* off3,
                         LookBackState lb, uint32_t* tile_counter, float* out, uint64_t cap,
                         unsigned long long* total, uint32_t* err, cudaStream_t st) {
    const unsigned tiles = (unsigned)((n + kThreads * 16 - 1) / (kThreads * 16));
    if (tiles) expand_cells_kernel<<<tiles, kThreads, 0, st>>>(cells, counts, n, q, off3, lb, tile_counter, out, cap, total, err);
}
void launch_quantize_cells(const float* xyz, uint64_t n, QuantParams q, const PointStats* stats, int32_t* cells,
                           cudaStream_t st) {
    quantize_cells_kernel<<<grid_for(n), kThreads, 0, st>>>(xyz, n, q, stats, cells);
}
void launch_recover_cells(const int32_t* cells, uint64_t n, QuantParams q, const float* offset3_dev, float* xyz,
                          cudaStream_t st) {
    recover_cells_kernel<<<grid_for(n), kThreads, 0, st>>>(cells, n, q, offset3_dev, xyz);
}
void launch_hilbert(const unsigned long long* in, uint64_t n, const uint8_t* tab, int top, unsigned int state,
                    unsigned long long* out, cudaStream_t st) {
    hilbert_kernel<<<grid_for(n), kThreads, 0, st>>>(in, n, tab, top, state, out);
}

}  // namespace dev
}  // namespace xnyz
