// The block-parameter predictor: a 34 -> 64 -> 64 -> (32 + 33) MLP whose dense layers run
// on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation).
//
//   x (34 features, zero-padded to 48) -> h1 = relu(W1 x + b1) -> h2 = relu(W2 h1 + b2)
//   -> logits = W3 h2 + b3: logits[0..31] score the Golomb-Rice k, logits[32..64] the PFor
//   width w (rows 65..71 of W3 are padding).
//
// Parameters are one FP32 array (the training master copy, layout kParam* in kernels.h);
// kernels round weights, activations and back-propagated gradients to BF16 for the MMAs.
// One warp handles 16 samples: the M dimension of the MMA.  Kernels:
//   * forward: logits, argmax per head and the head's softmax confidence;
//   * train: forward + softmax cross-entropy of both heads + backward; weight gradients are
//     MMAs too (dW = dY^T X over the warp's 16 samples), summed per CTA in shared memory and
//     added to the global FP32 gradient;
//   * adam: the update, which also clears the gradient.
#include <cuda_bf16.h>

#include "device_common.cuh"
#include "kernels.h"

namespace xnyz {
namespace dev {

namespace {

constexpr int NI = 48;   // padded input width (34 used)
constexpr int NH = 64;   // hidden width
constexpr int NO = 72;   // padded output width (65 used)
constexpr int NOP = 80;  // output width padded to a K multiple of 16 for the backward MMA
constexpr int WARPS = 4;
constexpr int THREADS = 32 * WARPS;
static_assert(kParamInputs == 34 && kParamOutputsK == 32 && kParamOutputsW == 33, "network shape");

// parameter offsets in the FP32 array
constexpr int oW1 = 0, ob1 = oW1 + NH * NI, oW2 = ob1 + NH, ob2 = oW2 + NH * NH, oW3 = ob2 + NH, ob3 = oW3 + NO * NH,
              oEnd = ob3 + NO;
static_assert(oEnd == kParamCount, "parameter count");

using bf16 = __nv_bfloat16;

__device__ __forceinline__ u32 pack2(bf16 lo, bf16 hi) {
    return (u32)__bfloat16_as_ushort(lo) | ((u32)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ u32 pack2f(float lo, float hi) { return pack2(__float2bfloat16_rn(lo), __float2bfloat16_rn(hi)); }

__device__ __forceinline__ void mma16816(float (&d)[4], u32 a0, u32 a1, u32 a2, u32 a3, u32 b0, u32 b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Operand accessors returning two consecutive BF16 elements packed (first in the low half).
// A(r, c): elements (r, c), (r, c + 1).  B(k, n): elements (k, n), (k + 1, n).
struct RowPairs {  // matrix M[r][c] with c contiguous: pairs along c
    const bf16* p;
    int ld;
    __device__ __forceinline__ u32 operator()(int r, int c) const {
        return *reinterpret_cast<const u32*>(p + r * ld + c);
    }
};
struct ColPairs {  // matrix M[r][c] stored as S[c][r]: pairs along c
    const bf16* p;
    int ld;
    __device__ __forceinline__ u32 operator()(int r, int c) const { return pack2(p[c * ld + r], p[(c + 1) * ld + r]); }
};

// acc[NT][4] (C[16][8*NT]) += A[16][16*KT] * B[16*KT][8*NT], A(r, c) row pairs, B given as
// Bt(n, k) pairs along k (Bt = B transposed).
template <int KT, int NT, class FA, class FB>
__device__ __forceinline__ void warp_gemm(float (&acc)[NT][4], const FA& A, const FB& Bt) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
        const int c0 = kt * 16 + 2 * t;
        const u32 a0 = A(g, c0), a1 = A(g + 8, c0), a2 = A(g, c0 + 8), a3 = A(g + 8, c0 + 8);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const u32 b0 = Bt(nt * 8 + g, c0), b1 = Bt(nt * 8 + g, c0 + 8);
            mma16816(acc[nt], a0, a1, a2, a3, b0, b1);
        }
    }
}

struct Weights {  // shared-memory BF16 copies
    bf16 W1[NH * NI];    // [out][in]
    bf16 W2[NH * NH];
    bf16 W3[NO * NH];
    bf16 W2T[NH * NH];   // [in][out]
    bf16 W3T[NH * NOP];  // [in][out], outputs padded to 80
    float b1[NH], b2[NH], b3[NO];
};

struct WarpTile {  // per-warp activations of 16 samples
    bf16 X[16 * NI];
    bf16 H1[16 * NH];
    bf16 H2[16 * NH];
    bf16 D3[16 * NOP];
    bf16 D2[16 * NH];
    bf16 D1[16 * NH];
    float L[16 * NO];
};

__device__ void load_weights(Weights& s, const float* __restrict__ prm, bool transposed) {
    for (int i = threadIdx.x; i < NH * NI; i += THREADS) s.W1[i] = __float2bfloat16_rn(prm[oW1 + i]);
    for (int i = threadIdx.x; i < NH * NH; i += THREADS) s.W2[i] = __float2bfloat16_rn(prm[oW2 + i]);
    for (int i = threadIdx.x; i < NO * NH; i += THREADS) s.W3[i] = __float2bfloat16_rn(prm[oW3 + i]);
    if (transposed) {
        for (int i = threadIdx.x; i < NH * NH; i += THREADS) {
            const int o = i / NH, in = i % NH;
            s.W2T[in * NH + o] = __float2bfloat16_rn(prm[oW2 + i]);
        }
        for (int i = threadIdx.x; i < NH * NOP; i += THREADS) {
            const int in = i / NOP, o = i % NOP;
            s.W3T[i] = __float2bfloat16_rn(o < NO ? prm[oW3 + o * NH + in] : 0.f);
        }
    }
    for (int i = threadIdx.x; i < NH; i += THREADS) {
        s.b1[i] = prm[ob1 + i];
        s.b2[i] = prm[ob2 + i];
    }
    for (int i = threadIdx.x; i < NO; i += THREADS) s.b3[i] = prm[ob3 + i];
}

// C-fragment element (row, col) positions of tile nt: (g, 8nt + 2t + j) and (g + 8, ...).
template <int NT>
__device__ __forceinline__ void store_act(bf16* dst, int ld, const float (&acc)[NT][4], const float* bias, bool relu) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
        const int c = nt * 8 + 2 * t;
        float v0 = acc[nt][0] + bias[c], v1 = acc[nt][1] + bias[c + 1];
        float v2 = acc[nt][2] + bias[c], v3 = acc[nt][3] + bias[c + 1];
        if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
            v2 = fmaxf(v2, 0.f);
            v3 = fmaxf(v3, 0.f);
        }
        *reinterpret_cast<u32*>(dst + g * ld + c) = pack2f(v0, v1);
        *reinterpret_cast<u32*>(dst + (g + 8) * ld + c) = pack2f(v2, v3);
    }
}

// Forward of the warp's 16 samples starting at s0 (rows past `count` use zero features).
__device__ void warp_forward(const Weights& s, WarpTile& w, const float* __restrict__ feats, u64 s0, u64 count) {
    const int lane = threadIdx.x & 31;
    for (int i = lane; i < 16 * NI; i += 32) {
        const int r = i / NI, c = i % NI;
        const u64 row = s0 + r;
        w.X[i] = __float2bfloat16_rn((row < count && c < kParamInputs) ? feats[row * kParamFeatures + c] : 0.f);
    }
    __syncwarp();
    {
        float acc[NH / 8][4] = {};
        warp_gemm<NI / 16, NH / 8>(acc, RowPairs{w.X, NI}, RowPairs{s.W1, NI});
        store_act<NH / 8>(w.H1, NH, acc, s.b1, true);
    }
    __syncwarp();
    {
        float acc[NH / 8][4] = {};
        warp_gemm<NH / 16, NH / 8>(acc, RowPairs{w.H1, NH}, RowPairs{s.W2, NH});
        store_act<NH / 8>(w.H2, NH, acc, s.b2, true);
    }
    __syncwarp();
    {
        float acc[NO / 8][4] = {};
        warp_gemm<NH / 16, NO / 8>(acc, RowPairs{w.H2, NH}, RowPairs{s.W3, NH});
        const int g = lane >> 2, t = lane & 3;
#pragma unroll
        for (int nt = 0; nt < NO / 8; ++nt) {
            const int c = nt * 8 + 2 * t;
            w.L[g * NO + c] = acc[nt][0] + s.b3[c];
            w.L[g * NO + c + 1] = acc[nt][1] + s.b3[c + 1];
            w.L[(g + 8) * NO + c] = acc[nt][2] + s.b3[c];
            w.L[(g + 8) * NO + c + 1] = acc[nt][3] + s.b3[c + 1];
        }
    }
    __syncwarp();
}

// Head of lane: row = lane & 15, head 0 (k: logits 0..31) or head 1 (w: logits 32..64).
__device__ __forceinline__ void head_range(int head, int& lo, int& n) {
    lo = head ? kParamOutputsK : 0;
    n = head ? kParamOutputsW : kParamOutputsK;
}

// Inference layout: row pitches of 56 and 72 bf16 (28 and 36 words), so the 8 row groups of
// an MMA fragment load fall in distinct banks; no backward tiles, so 12 warps of 16 samples
// fit twice per SM.
constexpr int LI = NI + 8;
constexpr int LH = NH + 8;
constexpr int FWARPS = 12;
constexpr int FTHREADS = 32 * FWARPS;

struct FwdShared {
    bf16 W1[NH * LI];  // [out][in]
    bf16 W2[NH * LH];
    bf16 W3[NO * LH];
    float b1[NH], b2[NH], b3[NO];
    struct Tile {
        bf16 X[16 * LI];
        bf16 H1[16 * LH];
        bf16 H2[16 * LH];
    } t[FWARPS];
};

// Argmax (first maximum, 0 when no logit exceeds -inf) and 1 / sum(exp(logit - max)) of
// one head for row g + 8 * half of the warp's C fragments, combined over the 4 lanes that
// hold the row.
template <int NT0, int NT1>
__device__ __forceinline__ void head_argmax(const float (&acc)[NO / 8][4], const float* b3, int half, int lo, int hi,
                                            int& am, float& conf) {
    const int t = threadIdx.x & 3;
    float m = -INFINITY;
    int a = 1 << 10;
#pragma unroll
    for (int nt = NT0; nt < NT1; ++nt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c = nt * 8 + 2 * t + j;
            const float v = acc[nt][2 * half + j] + b3[c];
            if (c < hi && v > m) {
                m = v;
                a = c - lo;
            }
        }
#pragma unroll
    for (int off = 1; off <= 2; off <<= 1) {
        const float om = __shfl_xor_sync(kFullMask, m, off);
        const int oa = __shfl_xor_sync(kFullMask, a, off);
        if (om > m || (om == m && oa < a)) {
            m = om;
            a = oa;
        }
    }
    float se = 0.f;
#pragma unroll
    for (int nt = NT0; nt < NT1; ++nt)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int c = nt * 8 + 2 * t + j;
            if (c < hi) se += __expf(acc[nt][2 * half + j] + b3[c] - m);
        }
    se += __shfl_xor_sync(kFullMask, se, 1);
    se += __shfl_xor_sync(kFullMask, se, 2);
    am = a == (1 << 10) ? 0 : a;
    conf = 1.0f / se;
}

__global__ void __launch_bounds__(FTHREADS) forward_kernel(const float* __restrict__ prm, const float* __restrict__ feats,
                                                           u64 count, u8* __restrict__ wout, u8* __restrict__ kout,
                                                           float* __restrict__ conf, float* __restrict__ logits) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FwdShared& s = *reinterpret_cast<FwdShared*>(smem_raw);
    for (int i = threadIdx.x; i < NH * NI; i += FTHREADS)
        s.W1[(i / NI) * LI + i % NI] = __float2bfloat16_rn(prm[oW1 + i]);
    for (int i = threadIdx.x; i < NH * NH; i += FTHREADS)
        s.W2[(i / NH) * LH + i % NH] = __float2bfloat16_rn(prm[oW2 + i]);
    for (int i = threadIdx.x; i < NO * NH; i += FTHREADS)
        s.W3[(i / NH) * LH + i % NH] = __float2bfloat16_rn(prm[oW3 + i]);
    for (int i = threadIdx.x; i < NH; i += FTHREADS) {
        s.b1[i] = prm[ob1 + i];
        s.b2[i] = prm[ob2 + i];
    }
    for (int i = threadIdx.x; i < NO; i += FTHREADS) s.b3[i] = prm[ob3 + i];
    __syncthreads();
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    FwdShared::Tile& w = s.t[wi];
    const u64 ntiles = (count + 15) / 16;
    for (u64 tile = (u64)blockIdx.x * FWARPS + wi; tile < ntiles; tile += (u64)gridDim.x * FWARPS) {
        const u64 s0 = tile * 16;
        for (int i = lane; i < 16 * NI; i += 32) {
            const int r = i / NI, c = i % NI;
            const u64 row = s0 + r;
            w.X[r * LI + c] =
                __float2bfloat16_rn((row < count && c < kParamInputs) ? feats[row * kParamFeatures + c] : 0.f);
        }
        __syncwarp();
        {
            float acc[NH / 8][4] = {};
            warp_gemm<NI / 16, NH / 8>(acc, RowPairs{w.X, LI}, RowPairs{s.W1, LI});
            store_act<NH / 8>(w.H1, LH, acc, s.b1, true);
        }
        __syncwarp();
        {
            float acc[NH / 8][4] = {};
            warp_gemm<NH / 16, NH / 8>(acc, RowPairs{w.H1, LH}, RowPairs{s.W2, LH});
            store_act<NH / 8>(w.H2, LH, acc, s.b2, true);
        }
        __syncwarp();
        float acc[NO / 8][4] = {};
        warp_gemm<NH / 16, NO / 8>(acc, RowPairs{w.H2, LH}, RowPairs{s.W3, LH});
        __syncwarp();  // X, H1, H2 are rewritten by the next tile
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const u64 row = s0 + g + 8 * half;
            int ak, aw;
            float ck, cw;
            head_argmax<0, kParamOutputsK / 8>(acc, s.b3, half, 0, kParamOutputsK, ak, ck);
            head_argmax<kParamOutputsK / 8, NO / 8>(acc, s.b3, half, kParamOutputsK, kParamOutputsK + kParamOutputsW,
                                                    aw, cw);
            if (row < count) {
                if (t == 0) kout[row] = (u8)ak;
                if (t == 1) wout[row] = (u8)aw;
                if (conf && t == 2) conf[row * 2] = ck;
                if (conf && t == 3) conf[row * 2 + 1] = cw;
                if (logits) {
#pragma unroll
                    for (int nt = 0; nt < NO / 8; ++nt)
#pragma unroll
                        for (int j = 0; j < 2; ++j) {
                            const int c = nt * 8 + 2 * t + j;
                            if (c < kParamOutputsK + kParamOutputsW)
                                logits[row * (kParamOutputsK + kParamOutputsW) + c] = acc[nt][2 * half + j] + s.b3[c];
                        }
                }
            }
        }
    }
}

// dW[M = 16 * MT][N = 8 * NT] += D^T X over the warp's 16 samples; D[s][m] (ld dld), X[s][n]
// (ld xld); accumulated into FP32 shared memory g[m][n] (m < mmax).
template <int MT, int NT>
__device__ __forceinline__ void warp_weight_grad(float* g, int mmax, const bf16* D, int dld, const bf16* X, int xld) {
    const int lane = threadIdx.x & 31, gq = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
        float acc[NT][4] = {};
        // A(r = m, c = s) = D[s][m]: pairs along s; Bt(n, k = s) = X[s][n]: pairs along s
        const ColPairs A{D + mt * 16, dld};
        const ColPairs Bt{X, xld};
        warp_gemm<1, NT>(acc, A, Bt);
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int n = nt * 8 + 2 * t, m0 = mt * 16 + gq, m1 = m0 + 8;
            if (m0 < mmax) {
                atomicAdd(&g[m0 * (NT * 8) + n], acc[nt][0]);
                atomicAdd(&g[m0 * (NT * 8) + n + 1], acc[nt][1]);
            }
            if (m1 < mmax) {
                atomicAdd(&g[m1 * (NT * 8) + n], acc[nt][2]);
                atomicAdd(&g[m1 * (NT * 8) + n + 1], acc[nt][3]);
            }
        }
    }
}

// Column sums of D[16][ld] for columns < nc into g[].
__device__ __forceinline__ void warp_bias_grad(float* g, const bf16* D, int ld, int nc) {
    const int lane = threadIdx.x & 31;
    for (int c = lane; c < nc; c += 32) {
        float s = 0.f;
        for (int r = 0; r < 16; ++r) s += __bfloat162float(D[r * ld + c]);
        atomicAdd(&g[c], s);
    }
}

// dH[16][64] = D[16][K] * W  (W[out = K][in = 64], given as WT[in][K]); the ReLU mask of the
// layer's output H gives dZ, stored as BF16.
template <int KT>
__device__ __forceinline__ void warp_backprop(bf16* dZ, const bf16* D, int dld, const bf16* WT, int wtld, const bf16* H) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    float acc[NH / 8][4] = {};
    warp_gemm<KT, NH / 8>(acc, RowPairs{D, dld}, RowPairs{WT, wtld});
#pragma unroll
    for (int nt = 0; nt < NH / 8; ++nt) {
        const int c = nt * 8 + 2 * t;
        const float m0 = __bfloat162float(H[g * NH + c]) > 0.f ? 1.f : 0.f;
        const float m1 = __bfloat162float(H[g * NH + c + 1]) > 0.f ? 1.f : 0.f;
        const float m2 = __bfloat162float(H[(g + 8) * NH + c]) > 0.f ? 1.f : 0.f;
        const float m3 = __bfloat162float(H[(g + 8) * NH + c + 1]) > 0.f ? 1.f : 0.f;
        *reinterpret_cast<u32*>(dZ + g * NH + c) = pack2f(acc[nt][0] * m0, acc[nt][1] * m1);
        *reinterpret_cast<u32*>(dZ + (g + 8) * NH + c) = pack2f(acc[nt][2] * m2, acc[nt][3] * m3);
    }
}

struct TrainShared {
    Weights s;
    float g[kParamCount];  // gradient of this CTA
    WarpTile tiles[WARPS];
};

// Samples idx[first .. first + count) (idx null: first + i).  grad += d(loss)/d(params),
// loss += sum of the two heads' cross-entropies, both scaled by `scale`.
__global__ void __launch_bounds__(THREADS) train_kernel(const float* __restrict__ prm, const float* __restrict__ feats,
                                                        const u8* __restrict__ wlab, const u8* __restrict__ klab,
                                                        const u32* __restrict__ idx, u64 first, u64 count, float scale,
                                                        float* __restrict__ grad, float* __restrict__ loss,
                                                        float* __restrict__ gather) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainShared& T = *reinterpret_cast<TrainShared*>(smem_raw);
    load_weights(T.s, prm, true);
    for (int i = threadIdx.x; i < kParamCount; i += THREADS) T.g[i] = 0.f;
    __syncthreads();
    const int wi = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpTile& w = T.tiles[wi];
    const u64 ntiles = (count + 15) / 16;
    float lsum = 0.f;
    // the warp's features are gathered through idx into `gather` (16 x 34 per warp slot)
    float* gf = gather + ((u64)blockIdx.x * WARPS + wi) * 16 * kParamFeatures;
    for (u64 tile = (u64)blockIdx.x * WARPS + wi; tile < ntiles; tile += (u64)gridDim.x * WARPS) {
        const u64 s0 = tile * 16;
        for (int i = lane; i < 16 * kParamFeatures; i += 32) {
            const u64 r = s0 + i / kParamFeatures;
            const u64 src = r < count ? (idx ? idx[first + r] : first + r) : 0ull;
            gf[i] = r < count ? feats[src * kParamFeatures + i % kParamFeatures] : 0.f;
        }
        __syncwarp();
        warp_forward(T.s, w, gf, 0, min((u64)16, count - s0));
        // softmax cross-entropy: lane -> (row, head)
        {
            const int r = lane & 15, head = lane >> 4;
            const u64 row = s0 + r;
            int lo, nn;
            head_range(head, lo, nn);
            const bool ok = row < count;
            int lab = 0;
            if (ok) {
                const u64 src = idx ? idx[first + row] : first + row;
                lab = head ? min((int)wlab[src], kParamOutputsW - 1) : min((int)klab[src], kParamOutputsK - 1);
            }
            float m = -INFINITY;
            for (int j = 0; j < nn; ++j) m = fmaxf(m, w.L[r * NO + lo + j]);
            float se = 0.f;
            for (int j = 0; j < nn; ++j) se += expf(w.L[r * NO + lo + j] - m);
            const float lse = m + logf(se);
            if (ok) lsum += (lse - w.L[r * NO + lo + lab]) * scale;
            for (int j = 0; j < nn; ++j) {
                const float p = expf(w.L[r * NO + lo + j] - lse);
                const float d = ok ? (p - (j == lab ? 1.f : 0.f)) * scale : 0.f;
                w.D3[r * NOP + lo + j] = __float2bfloat16_rn(d);
            }
            if (head == 1)
                for (int j = kParamOutputsK + kParamOutputsW; j < NOP; ++j) w.D3[r * NOP + j] = __float2bfloat16_rn(0.f);
        }
        __syncwarp();
        float* g = T.g;
        warp_weight_grad<NOP / 16, NH / 8>(g + oW3, NO, w.D3, NOP, w.H2, NH);
        warp_bias_grad(g + ob3, w.D3, NOP, NO);
        warp_backprop<NOP / 16>(w.D2, w.D3, NOP, T.s.W3T, NOP, w.H2);
        __syncwarp();
        warp_weight_grad<NH / 16, NH / 8>(g + oW2, NH, w.D2, NH, w.H1, NH);
        warp_bias_grad(g + ob2, w.D2, NH, NH);
        warp_backprop<NH / 16>(w.D1, w.D2, NH, T.s.W2T, NH, w.H1);
        __syncwarp();
        warp_weight_grad<NH / 16, NI / 8>(g + oW1, NH, w.D1, NH, w.X, NI);
        warp_bias_grad(g + ob1, w.D1, NH, NH);
        __syncwarp();
    }
    for (int d = 16; d > 0; d >>= 1) lsum += __shfl_xor_sync(kFullMask, lsum, d);
    if (lane == 0 && lsum != 0.f) atomicAdd(loss, lsum);
    __syncthreads();
    for (int i = threadIdx.x; i < kParamCount; i += THREADS)
        if (T.g[i] != 0.f) atomicAdd(&grad[i], T.g[i]);
}

__global__ void adam_kernel(float* __restrict__ prm, float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = grad[i];
        const float mi = b1 * m[i] + (1.f - b1) * g;
        const float vi = b2 * v[i] + (1.f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        grad[i] = 0.f;
    }
}

}  // namespace

size_t mlp_gather_floats(uint64_t count) {
    const u64 ntiles = (count + 15) / 16;
    u64 ctas = (ntiles + WARPS - 1) / WARPS;
    if (ctas > 148) ctas = 148;
    return (size_t)(ctas ? ctas : 1) * WARPS * 16 * kParamFeatures;
}

void launch_mlp_forward(const float* prm, const float* feats, uint64_t count, uint8_t* w, uint8_t* k, float* conf,
                        float* logits, cudaStream_t st) {
    if (!count) return;
    const int smem = (int)sizeof(FwdShared);
    cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const u64 ntiles = (count + 15) / 16;
    u64 ctas = (ntiles + FWARPS - 1) / FWARPS;
    if (ctas > 148 * 2) ctas = 148 * 2;  // two CTAs per SM (shared memory)
    forward_kernel<<<(unsigned)ctas, FTHREADS, smem, st>>>(prm, feats, count, w, k, conf, logits);
}

void launch_mlp_train(const float* prm, const float* feats, const uint8_t* wlab, const uint8_t* klab,
                      const uint32_t* idx, uint64_t first, uint64_t count, float scale, float* grad, float* loss,
                      float* gather, cudaStream_t st) {
    if (!count) return;
    const int smem = (int)sizeof(TrainShared);
    cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    const u64 ntiles = (count + 15) / 16;
    u64 ctas = (ntiles + WARPS - 1) / WARPS;
    if (ctas > 148) ctas = 148;
    train_kernel<<<(unsigned)ctas, THREADS, smem, st>>>(prm, feats, wlab, klab, idx, first, count, scale, grad, loss,
                                                        gather);
}

void launch_mlp_adam(float* prm, float* grad, float* m, float* v, float lr, int step, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    adam_kernel<<<(kParamCount + 255) / 256, 256, 0, st>>>(prm, grad, m, v, kParamCount, lr, b1, b2, 1e-8f, c1, c2);
}

}  // namespace dev
}  // namespace xnyz
