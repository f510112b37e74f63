// Device-side building blocks shared by the XnYZip sm_100a kernels:
//   * warp / block scans, decoupled look-back with bounded waits,
//   * exact float arithmetic of the quantizers (explicit _rn intrinsics, never contracted),
//   * Morton interleave and the table-driven Hilbert transform,
//   * warp-aggregated bit writers and bit readers for the MSB-first (Huffman,
//     exp-Golomb) and LSB-first (Golomb-Rice, bit-packing) streams.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace xnyz {

using u8 = uint8_t;
using u16 = uint16_t;
using u32 = uint32_t;
using u64 = unsigned long long;  // the type CUDA atomics take
using i32 = int32_t;
using i64 = long long;

constexpr u32 kFullMask = 0xffffffffu;

// Device error bits (OR-ed into a u32 the host reads after each stage).
constexpr u32 kErrTimeout = 1u;      // a bounded wait gave up
constexpr u32 kErrBadStream = 2u;    // a decoder ran past its input or found an invalid code
constexpr u32 kErrOverflow = 4u;     // an output bound was exceeded
constexpr u32 kErrPlacement = 8u;    // a scatter computed a position outside its array (skipped)

// Spin limit for look-back waits: ~1 s with the back-off below, then the waiting thread
// records kErrTimeout and proceeds with what it has (the host reports XNYZ_ERR_TIMEOUT).
constexpr u32 kSpinLimit = 1u << 23;

__device__ __forceinline__ u32 lanemask_lt() {
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}
__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }

// ------------------------------------------------------------------ scans ---------------
template <typename T, typename Op>
__device__ __forceinline__ T warp_inclusive(T v, Op op) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(kFullMask, v, d);
        if ((int)lane_id() >= d) v = op(o, v);
    }
    return v;
}

struct AddOp {
    template <typename T>
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
};

// Warp-wide inclusive sums over the 32 lanes.
template <typename T>
__device__ __forceinline__ T warp_incl_add(T v) {
    const u32 lane = lane_id();
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const T o = __shfl_up_sync(kFullMask, v, d);
        if (lane >= (u32)d) v += o;
    }
    return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFullMask, v, d);
    return v;
}

// Segmented inclusive sums over one round of 32 consecutive elements (lane order): lane i
// gets the sum of v over [h, i] with h the last head lane at or before i, or carry plus the
// sum over [0, i] when there is none (SegOp's semantics; carry = the running segment sum).
template <typename T>
__device__ __forceinline__ T warp_seg_incl(u32 heads, T v, T carry) {
    const T incl = warp_incl_add(v);
    const u32 le = heads & (lanemask_lt() | (1u << lane_id()));
    const T before = __shfl_sync(kFullMask, incl - v, le ? 31 - __clz(le) : 0);
    return le ? incl - before : carry + incl;
}

// Exclusive prefix over the block's warps of per-warp aggregates held in v[0..WARPS); the
// tile total goes to v[WARPS].  One thread.
template <int WARPS, typename T, typename Op>
__device__ __forceinline__ void warps_exclusive(T* v, T identity, Op op) {
    T run = identity;
    for (int i = 0; i < WARPS; ++i) {
        const T x = v[i];
        v[i] = run;
        run = op(run, x);
    }
    v[WARPS] = run;
}


// Block-wide exclusive scan (THREADS a multiple of 32, <= 1024).  `total` receives the
// block aggregate.  `scratch` holds THREADS/32 + 1 elements of shared memory.
template <int THREADS, typename T, typename Op>
__device__ __forceinline__ T block_exclusive(T v, T identity, Op op, T* scratch, T& total) {
    constexpr int W = THREADS / 32;
    const int w = threadIdx.x >> 5;
    T inc = warp_inclusive(v, op);
    if (lane_id() == 31) scratch[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = (int)lane_id() < W ? scratch[lane_id()] : identity;
        T si = warp_inclusive(s, op);
        if ((int)lane_id() < W) scratch[lane_id()] = si;  // inclusive over warps
    }
    __syncthreads();
    T warp_prefix = w == 0 ? identity : scratch[w - 1];
    T excl_in_warp = __shfl_up_sync(kFullMask, inc, 1);
    if (lane_id() == 0) excl_in_warp = identity;
    total = scratch[W - 1];
    T r = op(warp_prefix, excl_in_warp);
    __syncthreads();
    return r;
}

// ------------------------------------------------------------- look-back ----------------
// Single-pass chained scan state for one u64 channel: per tile a flag (0 empty,
// 1 aggregate published, 2 inclusive prefix published) and the two values.  Values are
// written before their flag with a fence in between; readers read the flag first.
struct LookBack64 {
    u32* flag;
    u64* agg;
    u64* inc;
};

__device__ __forceinline__ u32 ld_volatile(const u32* p) { return *(const volatile u32*)p; }
__device__ __forceinline__ u64 ld_volatile(const u64* p) { return *(const volatile u64*)p; }
__device__ __forceinline__ void st_volatile(u32* p, u32 v) { *(volatile u32*)p = v; }
__device__ __forceinline__ void st_volatile(u64* p, u64 v) { *(volatile u64*)p = v; }

// Generic single-thread look-back for an associative `op` over T (T is u64 or a small
// struct of u64 fields, accessed through load/store helpers).  Returns the exclusive
// prefix of `tile` and publishes its inclusive prefix.
template <typename T, typename Op, typename Load, typename Store>
__device__ T lookback(u32* flag, T* agg, T* inc, u32 tile, T mine, T identity, Op op, Load load, Store store,
                      u32* err) {
    if (tile == 0) {
        store(&inc[0], mine);
        __threadfence();
        st_volatile(&flag[0], 2u);
        return identity;
    }
    store(&agg[tile], mine);
    __threadfence();
    st_volatile(&flag[tile], 1u);
    T acc = identity;
    i64 t = (i64)tile - 1;
    u32 spins = 0;
    while (t >= 0) {
        u32 f = ld_volatile(&flag[t]);
        if (f == 0u) {
            if (++spins > kSpinLimit) {
                atomicOr(err, kErrTimeout);
                break;
            }
            if (spins > 64) __nanosleep(100);
            continue;
        }
        __threadfence();
        if (f == 2u) {
            acc = op(load(&inc[t]), acc);
            break;
        }
        acc = op(load(&agg[t]), acc);
        --t;
    }
    store(&inc[tile], op(acc, mine));
    __threadfence();
    st_volatile(&flag[tile], 2u);
    return acc;
}

struct LoadU64 {
    __device__ __forceinline__ u64 operator()(const u64* p) const { return ld_volatile(p); }
};
struct StoreU64 {
    __device__ __forceinline__ void operator()(u64* p, u64 v) const { st_volatile(p, v); }
};

__device__ __forceinline__ u64 lookback_add(LookBack64 lb, u32 tile, u64 mine, u32* err) {
    return lookback(lb.flag, lb.agg, lb.inc, tile, mine, (u64)0, AddOp{}, LoadU64{}, StoreU64{}, err);
}

// Segmented sum element: `head` = a segment starts inside, `sum` = sum since the last
// segment start (or of everything if no start).  combine(a, b) = a followed by b.
struct Seg {
    u64 head;  // 0 or 1
    u64 sum;
};
struct SegOp {
    __device__ __forceinline__ Seg operator()(Seg a, Seg b) const {
        return Seg{a.head | b.head, b.head ? b.sum : a.sum + b.sum};
    }
};
struct LoadSeg {
    __device__ __forceinline__ Seg operator()(const Seg* p) const {
        return Seg{ld_volatile(&p->head), ld_volatile(&p->sum)};
    }
};
struct StoreSeg {
    __device__ __forceinline__ void operator()(Seg* p, Seg v) const {
        st_volatile(&p->head, v.head);
        st_volatile(&p->sum, v.sum);
    }
};

// Warp-cooperative look-back: called by all 32 lanes of one warp, returns the exclusive
// prefix of `tile` to every lane and publishes its inclusive prefix.  Each step inspects 32
// predecessors at once (lane i: tile - 1 - i - 32 * step), waits until all of them have
// published something, then combines the aggregates up to the nearest inclusive prefix.
// `op` need not commute: earlier tiles are combined first.
__device__ __forceinline__ u64 shfl_down_t(u64 v, int d) { return __shfl_down_sync(kFullMask, v, d); }
__device__ __forceinline__ Seg shfl_down_t(Seg v, int d) {
    return Seg{__shfl_down_sync(kFullMask, v.head, d), __shfl_down_sync(kFullMask, v.sum, d)};
}
__device__ __forceinline__ u64 shfl_t(u64 v, int l) { return __shfl_sync(kFullMask, v, l); }
__device__ __forceinline__ Seg shfl_t(Seg v, int l) {
    return Seg{__shfl_sync(kFullMask, v.head, l), __shfl_sync(kFullMask, v.sum, l)};
}

template <typename T, typename Op, typename Load, typename Store>
__device__ T warp_lookback(u32* flag, T* agg, T* inc, u32 tile, T mine, T identity, Op op, Load load, Store store,
                           u32* err) {
    const int lane = (int)(threadIdx.x & 31u);
    if (tile == 0) {
        if (lane == 0) {
            store(&inc[0], mine);
            __threadfence();
            st_volatile(&flag[0], 2u);
        }
        __syncwarp();
        return identity;
    }
    if (lane == 0) {
        store(&agg[tile], mine);
        __threadfence();
        st_volatile(&flag[tile], 1u);
    }
    T acc = identity;
    i64 top = (i64)tile - 1;
    u32 spins = 0;
    bool failed = false;
    while (true) {
        const i64 p = top - lane;
        const u32 f = p >= 0 ? ld_volatile(&flag[p]) : 2u;
        if (__any_sync(kFullMask, f == 0u)) {
            if (++spins > kSpinLimit) {
                failed = true;
                break;
            }
            if (spins > 64) __nanosleep(100);
            continue;
        }
        __threadfence();
        T v = identity;
        if (p >= 0) v = f == 2u ? load(&inc[p]) : load(&agg[p]);
        const u32 m2 = __ballot_sync(kFullMask, f == 2u);
        const int last = m2 ? __ffs(m2) - 1 : 31;
        T r = lane <= last ? v : identity;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const T o = shfl_down_t(r, d);  // lane + d: an earlier tile
            if (lane + d < 32) r = op(o, r);
        }
        acc = op(shfl_t(r, 0), acc);
        if (m2) break;
        top -= 32;
    }
    if (lane == 0) {
        if (failed) atomicOr(err, kErrTimeout);
        store(&inc[tile], op(acc, mine));
        __threadfence();
        st_volatile(&flag[tile], 2u);
    }
    __syncwarp();
    return acc;
}

__device__ __forceinline__ u64 warp_lookback_add(LookBack64 lb, u32 tile, u64 mine, u32* err) {
    return warp_lookback(lb.flag, lb.agg, lb.inc, tile, mine, (u64)0, AddOp{}, LoadU64{}, StoreU64{}, err);
}

// Dynamic tile index: tiles are claimed in launch order, so a tile's predecessors have
// all started before it waits on them.
__device__ __forceinline__ u32 claim_tile(u32* counter, u32* smem_slot) {
    if (threadIdx.x == 0) *smem_slot = atomicAdd(counter, 1u);
    __syncthreads();
    return *smem_slot;
}

// ------------------------------------------------------------ quantizers ----------------
// Quantizer constants (dev::QuantParams) are derived on the host exactly as the reference
// derives them: div = float(double(2.0f * l2) / sqrt(5 or 3)) (quantize divisor), s = l2,
// rdiv = float(sqrt(5 or 3)) (recover: ((v * 2) * s) / rdiv).
using dev::QuantParams;

// static_cast<int>(float) as compiled for x86-64 (cvttss2si): truncation toward zero and
// 0x80000000 for NaN or values outside the int range.
__device__ __forceinline__ i32 f2i_x86(float f) {
    if (!(f > -2147483904.0f && f < 2147483648.0f)) return (i32)0x80000000;
    return __float2int_rz(f);
}

__device__ __forceinline__ float sqf(float a) { return __fmul_rn(a, a); }

// Truncated-octahedron (BCC) quantizer: nearest of the even and odd cubic lattices with
// the reference's coefficient-wise float operations, then x,y halved (quantizer/
// truncated_octahedron_quantizer.hpp:21-55).  squaredNorm sums as c0 + (c1 + c2).
__device__ __forceinline__ void quantize_to(float px, float py, float pz, float div, i32& ox, i32& oy, i32& oz) {
    const float q0 = __fdiv_rn(px, div), q1 = __fdiv_rn(py, div), q2 = __fdiv_rn(pz, div);
    const float e0 = __fmul_rn(roundf(__fmul_rn(q0, 0.5f)), 2.0f);
    const float e1 = __fmul_rn(roundf(__fmul_rn(q1, 0.5f)), 2.0f);
    const float e2 = __fmul_rn(roundf(__fmul_rn(q2, 0.5f)), 2.0f);
    const float o0 = __fadd_rn(__fmul_rn(roundf(__fmul_rn(__fsub_rn(q0, 1.0f), 0.5f)), 2.0f), 1.0f);
    const float o1 = __fadd_rn(__fmul_rn(roundf(__fmul_rn(__fsub_rn(q1, 1.0f), 0.5f)), 2.0f), 1.0f);
    const float o2 = __fadd_rn(__fmul_rn(roundf(__fmul_rn(__fsub_rn(q2, 1.0f), 0.5f)), 2.0f), 1.0f);
    const float dE = __fadd_rn(sqf(__fsub_rn(q0, e0)), __fadd_rn(sqf(__fsub_rn(q1, e1)), sqf(__fsub_rn(q2, e2))));
    const float dO = __fadd_rn(sqf(__fsub_rn(q0, o0)), __fadd_rn(sqf(__fsub_rn(q1, o1)), sqf(__fsub_rn(q2, o2))));
    i32 n0, n1, n2;
    if (dE <= dO) {
        n0 = f2i_x86(e0); n1 = f2i_x86(e1); n2 = f2i_x86(e2);
    } else {
        n0 = f2i_x86(o0); n1 = f2i_x86(o1); n2 = f2i_x86(o2);
    }
    if (n0 & 1) {
        n0 = (i32)((u32)n0 + 1u) >> 1;
        n1 = (i32)((u32)n1 + 1u) >> 1;
    } else {
        n0 >>= 1;
        n1 >>= 1;
    }
    ox = n0; oy = n1; oz = n2;
}

// Cube quantizer: floor(p / div) (quantizer/cube_quantizer.hpp:15-27).
__device__ __forceinline__ void quantize_cube(float px, float py, float pz, float div, i32& ox, i32& oy, i32& oz) {
    ox = f2i_x86(floorf(__fdiv_rn(px, div)));
    oy = f2i_x86(floorf(__fdiv_rn(py, div)));
    oz = f2i_x86(floorf(__fdiv_rn(pz, div)));
}

// Adaptive quantizer steps: from device memory while compressing, from the container's
// parameters while decompressing.
__device__ __forceinline__ float adaptive_step(const QuantParams& q, int a) {
    return q.step_dev ? q.step_dev[a] : q.step[a];
}

// Adaptive quantizer: round(p / step) per axis, half away from zero, then the x86 cast
// (quantizer/adaptive_quantizer.hpp:66-77).
__device__ __forceinline__ void quantize_adaptive(const QuantParams& q, float px, float py, float pz, i32& ox,
                                                  i32& oy, i32& oz) {
    ox = f2i_x86(roundf(__fdiv_rn(px, adaptive_step(q, 0))));
    oy = f2i_x86(roundf(__fdiv_rn(py, adaptive_step(q, 1))));
    oz = f2i_x86(roundf(__fdiv_rn(pz, adaptive_step(q, 2))));
}

__device__ __forceinline__ void quantize(const QuantParams& q, float px, float py, float pz, i32& ox, i32& oy,
                                         i32& oz) {
    if (q.quantizer == 1)
        quantize_to(px, py, pz, q.div, ox, oy, oz);
    else if (q.quantizer == 2)
        quantize_adaptive(q, px, py, pz, ox, oy, oz);
    else
        quantize_cube(px, py, pz, q.div, ox, oy, oz);
}

// Recover + unshift (truncated_octahedron_quantizer.hpp:57-76, cube_quantizer.hpp:29-38,
// adaptive_quantizer.hpp:83-97: idx * step, shifting.hpp:39-50).
__device__ __forceinline__ void recover(const QuantParams& q, i32 cx, i32 cy, i32 cz, float offx, float offy,
                                        float offz, float& x, float& y, float& z) {
    float fx, fy, fz;
    if (q.quantizer == 1) {
        i32 nx, ny;
        if (cz & 1) {
            nx = (i32)(((u32)cx << 1) - 1u);
            ny = (i32)(((u32)cy << 1) - 1u);
        } else {
            nx = (i32)((u32)cx << 1);
            ny = (i32)((u32)cy << 1);
        }
        fx = __fdiv_rn(__fmul_rn(__fmul_rn(__int2float_rn(nx), 2.0f), q.s), q.rdiv);
        fy = __fdiv_rn(__fmul_rn(__fmul_rn(__int2float_rn(ny), 2.0f), q.s), q.rdiv);
        fz = __fdiv_rn(__fmul_rn(__fmul_rn(__int2float_rn(cz), 2.0f), q.s), q.rdiv);
    } else if (q.quantizer == 2) {
        fx = __fmul_rn(__int2float_rn(cx), adaptive_step(q, 0));
        fy = __fmul_rn(__int2float_rn(cy), adaptive_step(q, 1));
        fz = __fmul_rn(__int2float_rn(cz), adaptive_step(q, 2));
    } else {
        fx = __fdiv_rn(__fmul_rn(__fmul_rn(__fadd_rn(__int2float_rn(cx), 0.5f), 2.0f), q.s), q.rdiv);
        fy = __fdiv_rn(__fmul_rn(__fmul_rn(__fadd_rn(__int2float_rn(cy), 0.5f), 2.0f), q.s), q.rdiv);
        fz = __fdiv_rn(__fmul_rn(__fmul_rn(__fadd_rn(__int2float_rn(cz), 0.5f), 2.0f), q.s), q.rdiv);
    }
    x = __fadd_rn(fx, offx);
    y = __fadd_rn(fy, offy);
    z = __fadd_rn(fz, offz);
}

// ------------------------------------------------------------------ Morton ---------------
// 21 bits per axis interleaved x (bit 0), y (bit 1), z (bit 2) (preprocessor/
// z_order_curve.hpp:14-47), with the usual mask cascade.
__device__ __forceinline__ u64 spread3(u32 v) {
    u64 x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}
__device__ __forceinline__ u32 gather3(u64 m) {
    u64 x = m & 0x1249249249249249ull;
    x = (x | (x >> 2)) & 0x10c30c30c30c30c3ull;
    x = (x | (x >> 4)) & 0x100f00f00f00f00full;
    x = (x | (x >> 8)) & 0x001f0000ff0000ffull;
    x = (x | (x >> 16)) & 0x001f00000000ffffull;
    x = (x | (x >> 32)) & 0x1fffffull;
    return (u32)x;
}
__device__ __forceinline__ u64 morton3(i32 x, i32 y, i32 z) {
    return spread3((u32)x) | (spread3((u32)y) << 1) | (spread3((u32)z) << 2);
}

// ------------------------------------------------------------------ Hilbert --------------
// Table-driven digit transform.  A state is one orientation of the curve (an element of
// the cube's rotation group, <= 32 states); entry [state*8 + digit] holds the output digit
// in bits 0-2 and the next state in bits 3-7.  Levels above `top` are left unchanged, as
// in mortonToHilbert3 / hilbertToMorton3 with iteration = top.
__device__ __forceinline__ u64 hilbert_apply(const u8* tab, u64 code, int top, u32 state) {
    u64 out = top >= 20 ? (code & (top >= 21 ? 0ull : ~0ull << 63)) : (code & (~0ull << (3 * (top + 1))));
    for (int l = top; l >= 0; --l) {
        const u32 d = (u32)(code >> (3 * l)) & 7u;
        const u32 e = tab[state * 8 + d];
        out |= (u64)(e & 7u) << (3 * l);
        state = e >> 3;
    }
    return out;
}

// gather3 of hilbert_apply(tab, code, top, state) for each axis: the output digit of level
// l is bit l of x, y and z (bits 0, 1, 2 of the digit), so the transformed levels are
// de-interleaved as they are produced; levels above `top` pass through gather3.
__device__ __forceinline__ void hilbert_xyz(const u8* tab, u64 code, int top, u32 state, u32& x, u32& y, u32& z) {
    const u64 above = top >= 20 ? (code & (top >= 21 ? 0ull : ~0ull << 63)) : (code & (~0ull << (3 * (top + 1))));
    x = y = z = 0;
    if (above) {
        x = gather3(above);
        y = gather3(above >> 1);
        z = gather3(above >> 2);
    }
    for (int l = top; l >= 0; --l) {
        const u32 e = tab[state * 8 + ((u32)(code >> (3 * l)) & 7u)];
        x |= (e & 1u) << l;
        y |= ((e >> 1) & 1u) << l;
        z |= ((e >> 2) & 1u) << l;
        state = e >> 3;
    }
}

// hilbert_xyz for top = 5 and a code below 2^18 (the 6 levels of one 64^3 quadrant).
__device__ __forceinline__ void hilbert_xyz6(const u8* tab, u32 code, u32 state, u32& x, u32& y, u32& z) {
    x = y = z = 0;
#pragma unroll
    for (int l = 5; l >= 0; --l) {
        const u32 e = tab[state * 8 + ((code >> (3 * l)) & 7u)];
        x |= (e & 1u) << l;
        y |= ((e >> 1) & 1u) << l;
        z |= ((e >> 2) & 1u) << l;
        state = e >> 3;
    }
}

// hilbert_apply(tab, morton3(x, y, z), 5, state) for x, y, z below 64: the input digit of
// level l is bit l of x, y and z, so the interleave is done as the levels are consumed.
__device__ __forceinline__ u32 hilbert_code6(const u8* tab, u32 x, u32 y, u32 z, u32 state) {
    u32 out = 0;
#pragma unroll
    for (int l = 5; l >= 0; --l) {
        const u32 d = ((x >> l) & 1u) | (((y >> l) & 1u) << 1) | (((z >> l) & 1u) << 2);
        const u32 e = tab[state * 8 + d];
        out |= (e & 7u) << (3 * l);
        state = e >> 3;
    }
    return out;
}

// ------------------------------------------------------------- bit writers --------------
// Stream words are 32-bit; the output buffer must be zeroed and 4-byte aligned.
// MSB-first streams: stream bit p is bit (7 - p%8) of byte p/8; a 32-bit word k then holds
// stream bits [32k, 32k+32) most significant first, stored byte-swapped in memory.
// LSB-first streams: stream bit p is bit p%8 of byte p/8 = bit p%32 of little-endian word k.
//
// Every lane of a warp calls these together (inactive lanes pass nbits = 0).  Lanes must
// pass non-decreasing positions in lane order (true for scan-derived offsets); the writes
// of lanes landing in the same word are OR-combined with shuffles first, so one atomicOr
// per distinct word and warp reaches memory.
__device__ __forceinline__ void warp_or_word(u32* words, u64 word, u32 bits, bool active) {
    // Segmented OR over lanes with equal `word` (non-decreasing across lanes).
    const u32 lane = lane_id();
    const int act = active ? 1 : 0;
    u32 v = active ? bits : 0u;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        u32 ov = __shfl_up_sync(kFullMask, v, d);
        u64 ow = __shfl_up_sync(kFullMask, word, d);
        int oa = __shfl_up_sync(kFullMask, act, d);
        if ((int)lane >= d && oa && ow == word) v |= ov;
    }
    u64 nw = __shfl_down_sync(kFullMask, word, 1);
    int na = __shfl_down_sync(kFullMask, act, 1);
    bool last = (lane == 31) || !na || nw != word;
    if (active && last && v) atomicOr(&words[word], v);
}

// Writes `nbits` (<= 64) bits of `val` (its low bits, most significant first) at stream
// position `pos` of an MSB-first stream.
__device__ __forceinline__ void warp_write_msb(u32* words, u64 pos, u64 val, u32 nbits) {
    const bool act = nbits != 0;
    const u64 k0 = pos >> 5;
    const u32 o = (u32)(pos & 31u);
    // 96-bit window W[k0] W[k0+1] W[k0+2]; the value occupies [o, o + nbits).
    unsigned __int128 chunk = 0;
    if (act) {
        const u64 v = nbits == 64 ? val : (val & ((1ull << nbits) - 1));
        chunk = (unsigned __int128)v << (96u - o - nbits);
    }
    const u32 w0 = (u32)(chunk >> 64), w1 = (u32)(chunk >> 32), w2 = (u32)chunk;
    warp_or_word(words, k0, __byte_perm(w0, 0, 0x0123), act);
    if (__any_sync(kFullMask, act && w1 != 0u)) warp_or_word(words, k0 + 1, __byte_perm(w1, 0, 0x0123), act);
    if (__any_sync(kFullMask, act && w2 != 0u)) warp_or_word(words, k0 + 2, __byte_perm(w2, 0, 0x0123), act);
}

// One thread's run of consecutive codes of an MSB-first stream, from stream bit `pos` on
// (begin / put / end).  Bits collect in a 64-bit buffer and leave a word at a time: the
// run's first and last words may be shared with the neighbouring runs and are OR-ed in
// atomically, the words in between belong to this run alone and are stored.  For short codes
// this is one or two memory operations per run instead of one per code.
struct MsbRun {
    u32* words;
    u64 k;    // word that buf's first bit belongs to
    u64 buf;  // pending bits, first in bit 63
    u32 nb;   // pending bits (< 32 between puts)
    bool first;
    __device__ __forceinline__ void begin(u32* w, u64 pos) {
        words = w;
        k = pos >> 5;
        nb = (u32)(pos & 31u);  // the word's leading bits belong to the previous run: zeros here
        buf = 0;
        first = true;
    }
    __device__ __forceinline__ void flush() {
        const u32 wv = __byte_perm((u32)(buf >> 32), 0, 0x0123);
        if (first) {
            if (wv) atomicOr(&words[k], wv);
            first = false;
        } else {
            words[k] = wv;
        }
        buf <<= 32;
        nb -= 32;
        ++k;
    }
    // the low n (<= 32) bits of v, most significant first
    __device__ __forceinline__ void put32(u32 v, u32 n) {
        if (!n) return;
        if (nb >= 32) flush();
        buf |= ((u64)v << (64u - n)) >> nb;
        nb += n;
    }
    __device__ __forceinline__ void zeros(u64 n) {
        while (n) {
            const u32 t = n > 32 ? 32u : (u32)n;
            put32(0u, t);
            n -= t;
        }
    }
    // the low n (<= 64) bits of v, most significant first
    __device__ __forceinline__ void put(u64 v, u32 n) {
        if (n > 32) {
            put32((u32)(v >> 32), n - 32);
            put32((u32)v, 32);
        } else {
            put32((u32)v, n);
        }
    }
    __device__ __forceinline__ void end() {
        if (nb >= 32) flush();
        if (nb) {  // the last word, shared with the next run
            const u32 wv = __byte_perm((u32)(buf >> 32), 0, 0x0123);
            if (wv) atomicOr(&words[k], wv);
        }
    }
};

// The LSB-first counterpart of MsbRun: bits collect from bit 0 of the buffer up.
struct LsbRun {
    u32* words;
    u64 k;
    u64 buf;  // pending bits, first in bit 0
    u32 nb;
    bool first;
    __device__ __forceinline__ void begin(u32* w, u64 pos) {
        words = w;
        k = pos >> 5;
        nb = (u32)(pos & 31u);
        buf = 0;
        first = true;
    }
    __device__ __forceinline__ void flush() {
        const u32 wv = (u32)buf;
        if (first) {
            if (wv) atomicOr(&words[k], wv);
            first = false;
        } else {
            words[k] = wv;
        }
        buf >>= 32;
        nb -= 32;
        ++k;
    }
    // the low n (<= 32) bits of v, least significant first
    __device__ __forceinline__ void put32(u32 v, u32 n) {
        if (!n) return;
        if (nb >= 32) flush();
        buf |= (u64)(n == 32u ? v : (v & ((1u << n) - 1u))) << nb;
        nb += n;
    }
    __device__ __forceinline__ void ones(u64 n) {
        while (n) {
            const u32 t = n > 32 ? 32u : (u32)n;
            put32(0xffffffffu, t);
            n -= t;
        }
    }
    __device__ __forceinline__ void put(u64 v, u32 n) {
        if (n > 32) {
            put32((u32)v, 32);
            put32((u32)(v >> 32), n - 32);
        } else {
            put32((u32)v, n);
        }
    }
    __device__ __forceinline__ void end() {
        if (nb >= 32) flush();
        if (nb) {
            const u32 wv = (u32)buf;
            if (wv) atomicOr(&words[k], wv);
        }
    }
};

// Writes `nbits` (<= 64) bits of `val`, least significant first, at position `pos` of an
// LSB-first stream.
__device__ __forceinline__ void warp_write_lsb(u32* words, u64 pos, u64 val, u32 nbits) {
    const bool act = nbits != 0;
    const u64 k0 = pos >> 5;
    const u32 o = (u32)(pos & 31u);
    unsigned __int128 chunk = 0;
    if (act) {
        const u64 v = nbits == 64 ? val : (val & ((1ull << nbits) - 1));
        chunk = (unsigned __int128)v << o;
    }
    const u32 w0 = (u32)chunk, w1 = (u32)(chunk >> 32), w2 = (u32)(chunk >> 64);
    warp_or_word(words, k0, w0, act);
    if (__any_sync(kFullMask, act && w1 != 0u)) warp_or_word(words, k0 + 1, w1, act);
    if (__any_sync(kFullMask, act && w2 != 0u)) warp_or_word(words, k0 + 2, w2, act);
}

// Single-lane writer of `count` one-bits at `pos` of an LSB-first stream (long unary runs
// of the Golomb-Rice code).  Whole words inside the run belong to this run alone.
__device__ __forceinline__ void write_ones_lsb(u32* words, u64 pos, u64 count) {
    while (count > 0) {
        const u64 k = pos >> 5;
        const u32 o = (u32)(pos & 31u);
        const u32 take = (u32)min((u64)(32u - o), count);
        const u32 mask = (take == 32u ? 0xffffffffu : ((1u << take) - 1u)) << o;
        if (mask == 0xffffffffu)
            words[k] = 0xffffffffu;
        else
            atomicOr(&words[k], mask);
        pos += take;
        count -= take;
    }
}

// ------------------------------------------------------------- bit readers --------------
// Streams are padded with >= 16 zero bytes so these may read past the last word.
__device__ __forceinline__ u32 load_be_word(const u32* w, u64 k) { return __byte_perm(__ldg(&w[k]), 0, 0x0123); }

// 32 bits of an MSB-first stream starting at bit `pos`, first bit in bit 31.
__device__ __forceinline__ u32 peek_msb32(const u32* w, u64 pos) {
    const u64 k = pos >> 5;
    const u32 o = (u32)(pos & 31u);
    const u32 a = load_be_word(w, k), b = load_be_word(w, k + 1);
    return o ? ((a << o) | (b >> (32u - o))) : a;
}
// 64 bits of an LSB-first stream starting at bit `pos`, first bit in bit 0.
__device__ __forceinline__ u64 peek_lsb64(const u32* w, u64 pos) {
    const u64 k = pos >> 5;
    const u32 o = (u32)(pos & 31u);
    const u64 a = __ldg(&w[k]), b = __ldg(&w[k + 1]), c = __ldg(&w[k + 2]);
    const unsigned __int128 x = (unsigned __int128)a | ((unsigned __int128)b << 32) | ((unsigned __int128)c << 64);
    return (u64)(x >> o);
}

__device__ __forceinline__ u32 bitlen64(u64 v) { return v ? 64u - (u32)__clzll((long long)v) : 0u; }

}  // namespace xnyz
