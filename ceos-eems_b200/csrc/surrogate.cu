// surrogate.cu -- learned constitutive surrogate for the FE^2 micro problems.
//
// No reference counterpart: CEOS obtains the homogenized response of a macro Gauss point by
// solving its RVE (MultiScale/ModMultiscaleAnalysis.f90:445-470).  Here an MLP energy
//   e(x),  x = [(C11-1, C22-1, C33-1, C12, C23, C13)/s_C, (vf - vf0)/s_vf],
//   z1 = W1 x + b1, h_l = softplus(z_l), z_l = W_l h_{l-1} + b_l (l = 2..4), e = w5.h4 + b5
// (width 128) stands in for the RVE solve.  S_k = a_k (s_W/s_C) de/dx_k, a = (2,2,2,1,1,1),
// and the material tangent C_pq = a_p a_q (s_W/s_C^2) d2e/dx_p dx_q.
//
// Training fits the stress (a Sobolev loss on de/dx, L = (1/N) sum w_k (g_k - t_k)^2) by the
// forward-over-reverse product d/dtheta (u.g), u = dL/dg, in four passes over the layers plus
// the weight gradients, every 128-wide contraction on the tensor cores in BF16 with FP32
// accumulation: forward primal, backward primal (gives g and u), forward tangent along u,
// backward tangent, then dW = a h^T + delta hdot^T.  The default path (tcgen05, TMEM
// accumulators) runs the four passes of 128 samples in one CTA of one launch (grad_chain_kernel);
// the mma.sync.m16n8k16 path launches one kernel per layer.  FP32 master weights and Adam; BF16
// copies (and transposed copies) of W1..W4 are refreshed after every step.
//
// Inference (FP32, CUDA cores) gives S and the 6x6 tangent per point from one forward pass,
// one backward pass and one forward pass of the Jacobians J_l = dz_l/dx accumulating
// d2e/dx2 = sum_l J_l^T diag(G_l sigma'(z_l)) J_l (G_l = de/dh_l), then pushes both forward to
// the Cauchy stress and the spatial tangent the element loop consumes.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/ceos_gpu.h"

namespace {

constexpr int kH = 128;      // hidden width
constexpr int kIn = 7;       // network inputs
constexpr int kInPad = 16;   // input width padded to one MMA k-step
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kH, oW4 = oB3 + kH, oB4 = oW4 + kH * kH, oW5 = oB4 + kH, oB5 = oW5 + kH,
              kNParams = oB5 + 1;
// offsets of W_l and b_l (layer index l = 0..3) in the parameter vector
__host__ __device__ constexpr int layer_w(int l) { return l == 0 ? oW1 : oW2 + (l - 1) * (kH * kH + kH); }
__host__ __device__ constexpr int layer_b(int l) { return l == 0 ? oB1 : oB2 + (l - 1) * (kH * kH + kH); }
static_assert(layer_w(3) == oW4 && layer_b(3) == oB4, "parameter layout");
constexpr int kTileN = 32;   // samples per CTA of the layer GEMMs
constexpr int kChunk = 256;  // samples per CTA of the weight-gradient GEMMs
constexpr int kTab = 513;    // vf grid of the reference-state stress table

__device__ __forceinline__ float softplus_f(float z) { return fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))); }
__device__ __forceinline__ float sigmoid_f(float z) { return 0.5f * (1.f + tanhf(0.5f * z)); }
// Training epilogues: the same functions from the fast exponential and logarithm (relative error
// about 1e-6, far below the BF16 rounding of the activations they produce); inference keeps the
// accurate ones above.
__device__ __forceinline__ float softplus_t(float z) { return fmaxf(z, 0.f) + __logf(1.f + __expf(-fabsf(z))); }
__device__ __forceinline__ float sigmoid_t(float z) { return __fdividef(1.f, 1.f + __expf(-z)); }

__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}
__device__ __forceinline__ uint4 pack_bf8(const float* x) {
    uint4 u;
    u.x = pack2(__float2bfloat16_rn(x[0]), __float2bfloat16_rn(x[1]));
    u.y = pack2(__float2bfloat16_rn(x[2]), __float2bfloat16_rn(x[3]));
    u.z = pack2(__float2bfloat16_rn(x[4]), __float2bfloat16_rn(x[5]));
    u.w = pack2(__float2bfloat16_rn(x[6]), __float2bfloat16_rn(x[7]));
    return u;
}

// ---------------------------------------------------------------------------------------------
// Layer GEMM: out[n][m] = sum_k Wop[m][k] in[n][k] (m < 128, k < K), n over a batch of samples.
// CTA = 4 warps, 32 samples; warp w owns rows [32w, 32w+32) x all 32 columns (8 MMA tiles).
// ---------------------------------------------------------------------------------------------
enum Epi { kFwd = 0, kBwd = 1, kFwdT = 2, kBwdT = 3 };

struct LayerArgs {
    int n;                        // samples
    const __nv_bfloat16* W;       // [128][K] row-major operand
    const __nv_bfloat16* in;      // [n][K]
    const float* bias;            // kFwd: b_l
    const float* w5;              // kFwd / kFwdT of the last layer: w5
    float* Z;                     // kFwd: z_l out;  kFwdT, kBwd, kBwdT: z of the layer (in)
    float* Zd;                    // kFwdT: zdot_l out; kBwdT: zdot of the layer (in)
    float* G;                     // kBwd: G out; kBwdT: G of the layer (in)
    __nv_bfloat16* outb;          // kFwd: h_l; kBwd: delta; kFwdT: hdot; kBwdT: a
    __nv_bfloat16* outb2;         // last layer: kFwd: delta_4 = sigma(z4) w5; kFwdT: a_4
    float* outf;                  // last layer kFwdT: hdot_4 in FP32 (for dw5)
    int last;                     // layer 4 (index 3)
    unsigned char* smem_next;     // chain kernel: the next layer's activation operand in shared memory,
                                  // written by the epilogue beside its global copy (null: global only)
    int n0;                       // chain kernel: first sample of the CTA (row 0 of smem_next)
};

// The 16-byte row chunk of 8 consecutive outputs m0.. of sample n in the canonical K-major operand
// layout (8-row x 16-byte core matrices, K chunks 128 bytes apart, 8-row groups 2048 bytes apart).
__device__ __forceinline__ void st_next(const LayerArgs& A, int n, int m0, uint4 u) {
    if (A.smem_next) {
        const int r = n - A.n0;
        *reinterpret_cast<uint4*>(A.smem_next + (r >> 3) * 2048 + (m0 >> 3) * 128 + (r & 7) * 16) = u;
    }
}
// 8 BF16 outputs m0.. of sample n to global memory and, when they are the next layer's input, to its
// shared-memory operand as well
__device__ __forceinline__ void st_out8(const LayerArgs& A, __nv_bfloat16* dst, const float* x, int n, int m0,
                                        bool next) {
    const uint4 u = pack_bf8(x);
    *reinterpret_cast<uint4*>(dst) = u;
    if (next) st_next(A, n, m0, u);
}

template <int K, int EPI>
__global__ void __launch_bounds__(128) layer_gemm_kernel(LayerArgs A) {
    constexpr int LDS = K + 8;  // padded row (bf16 elements): conflict-free fragment loads
    __shared__ __align__(16) __nv_bfloat16 Ws[kH * LDS];
    __shared__ __align__(16) __nv_bfloat16 Is[kTileN * LDS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    const int n0 = blockIdx.x * kTileN;
    constexpr int CPR = K / 8;  // 16-byte chunks per row
    for (int c = tid; c < kH * CPR; c += 128) {
        const int r = c / CPR, q = c - r * CPR;
        *reinterpret_cast<uint4*>(Ws + r * LDS + q * 8) = *reinterpret_cast<const uint4*>(A.W + (size_t)r * K + q * 8);
    }
    for (int c = tid; c < kTileN * CPR; c += 128) {
        const int r = c / CPR, q = c - r * CPR;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (n0 + r < A.n) v = *reinterpret_cast<const uint4*>(A.in + (size_t)(n0 + r) * K + q * 8);
        *reinterpret_cast<uint4*>(Is + r * LDS + q * 8) = v;
    }
    __syncthreads();
    constexpr int NT = kTileN / 8;
    float acc[2][NT][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[i][j][k] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
        uint32_t af[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r0 = 32 * warp + 16 * mt;
            af[mt][0] = *reinterpret_cast<const uint32_t*>(Ws + (r0 + g) * LDS + k0 + 2 * t);
            af[mt][1] = *reinterpret_cast<const uint32_t*>(Ws + (r0 + g + 8) * LDS + k0 + 2 * t);
            af[mt][2] = *reinterpret_cast<const uint32_t*>(Ws + (r0 + g) * LDS + k0 + 2 * t + 8);
            af[mt][3] = *reinterpret_cast<const uint32_t*>(Ws + (r0 + g + 8) * LDS + k0 + 2 * t + 8);
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            uint32_t bf[2];
            bf[0] = *reinterpret_cast<const uint32_t*>(Is + (8 * nt + g) * LDS + k0 + 2 * t);
            bf[1] = *reinterpret_cast<const uint32_t*>(Is + (8 * nt + g) * LDS + k0 + 2 * t + 8);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma_bf16(acc[mt][nt], af[mt], bf);
        }
    }
    // epilogue: accumulator (mt, nt, q) is row m = 32w + 16mt + g + 8(q>>1), column 8nt + 2t + (q&1)
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int m = 32 * warp + 16 * mt + g + 8 * (q >> 1);
                const int n = n0 + 8 * nt + 2 * t + (q & 1);
                if (n >= A.n) continue;
                const size_t o = (size_t)n * kH + m;
                const float v = acc[mt][nt][q];
                if constexpr (EPI == kFwd) {
                    const float z = v + A.bias[m];
                    A.Z[o] = z;
                    A.outb[o] = __float2bfloat16_rn(softplus_t(z));
                    if (A.last) A.outb2[o] = __float2bfloat16_rn(sigmoid_t(z) * A.w5[m]);
                } else if constexpr (EPI == kBwd) {
                    A.G[o] = v;
                    A.outb[o] = __float2bfloat16_rn(sigmoid_t(A.Z[o]) * v);
                } else if constexpr (EPI == kFwdT) {
                    A.Zd[o] = v;
                    const float s = sigmoid_t(A.Z[o]);
                    if (A.last) {
                        A.outf[o] = s * v;
                        A.outb2[o] = __float2bfloat16_rn(s * (1.f - s) * v * A.w5[m]);
                    } else {
                        A.outb[o] = __float2bfloat16_rn(s * v);
                    }
                } else {
                    const float s = sigmoid_t(A.Z[o]);
                    A.outb[o] = __float2bfloat16_rn(s * v + s * (1.f - s) * A.Zd[o] * A.G[o]);
                }
            }
}

// ---------------------------------------------------------------------------------------------
// The same 128-wide layer GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
// CTA = 128 threads, 128 samples x 128 outputs: D[n][m] = sum_k in[n][k] W[m][k] with
//   A = in  (M = 128 samples x K = 128, K-major),  B = W (N = 128 outputs x K = 128, K-major),
// both staged in shared memory in the canonical K-major layout without swizzle (8-row x 16-byte
// core matrices; the two 8-element K halves of one MMA step 128 bytes apart, 8-row groups 2048
// bytes apart), one thread issuing the 8 tcgen05.mma of K = 16 (BF16 in, FP32 accumulate in
// tensor memory) and committing them to an mbarrier, then each warp reading its 32 TMEM lanes
// (samples) with tcgen05.ld and running the layer's epilogue on 8 outputs at a time.
// ---------------------------------------------------------------------------------------------
constexpr int kUmmaRows = 128;                 // samples per CTA (M) and outputs (N)
constexpr int kUmmaOpBytes = 128 * 128 * 2;    // one 128 x 128 BF16 operand
constexpr unsigned long long kUmmaWaitNs = 100ull * 1000 * 1000;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, leading byte offset 128 (the next 8 K
// elements), stride byte offset 2048 (the next 8 rows), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(2048 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;  // base offset 0, layout type 0 (no swizzle)
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major, N = 128, M = 128.
constexpr uint32_t kUmmaIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(128 >> 3) << 17) |
                                ((uint32_t)(128 >> 4) << 24);

__device__ __forceinline__ void cp_async16_zfill(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(valid ? 16 : 0));
}

// The epilogue of 32 consecutive outputs m0..m0+31 of sample n: every FP32 input of the chunk (z,
// zdot, G of the layer, as the pass needs) is loaded before any of it is used, so a chunk costs one
// memory latency rather than one per group of 8 (the stores of a group could alias the loads of the
// next, so the compiler cannot hoist them itself).
template <int EPI>
__device__ __forceinline__ void layer_epilogue32(const LayerArgs& A, int n, int m0, const float* v);

// The epilogue of 8 outputs of the forward passes (layer 1 on the CUDA cores, and the forward primal
// groups of layer_epilogue32); the backward passes only run through layer_epilogue32.
template <int EPI>
__device__ __forceinline__ void layer_epilogue8(const LayerArgs& A, int n, int m0, const float* v) {
    static_assert(EPI == kFwd || EPI == kFwdT, "forward passes only");
    const size_t o = (size_t)n * kH + m0;
    auto ld8 = [](const float* src, float* x) {
        const float4 a = *reinterpret_cast<const float4*>(src), b = *reinterpret_cast<const float4*>(src + 4);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    };
    auto st8 = [](float* dst, const float* x) {
        *reinterpret_cast<float4*>(dst) = make_float4(x[0], x[1], x[2], x[3]);
        *reinterpret_cast<float4*>(dst + 4) = make_float4(x[4], x[5], x[6], x[7]);
    };
    float a[8], b[8];
    if constexpr (EPI == kFwd) {
        float z[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) z[j] = v[j] + A.bias[m0 + j];
        st8(A.Z + o, z);
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = softplus_t(z[j]);
        st_out8(A, A.outb + o, a, n, m0, !A.last);
        if (A.last) {
#pragma unroll
            for (int j = 0; j < 8; ++j) b[j] = sigmoid_t(z[j]) * A.w5[m0 + j];
            st_out8(A, A.outb2 + o, b, n, m0, true);
        }
    } else {
        float z[8];
        ld8(A.Z + o, z);
        st8(A.Zd + o, v);
        if (A.last) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float sg = sigmoid_t(z[j]);
                a[j] = sg * v[j];
                b[j] = sg * (1.f - sg) * v[j] * A.w5[m0 + j];
            }
            st8(A.outf + o, a);
            st_out8(A, A.outb2 + o, b, n, m0, true);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) a[j] = sigmoid_t(z[j]) * v[j];
            st_out8(A, A.outb + o, a, n, m0, true);
        }
    }
}

template <int EPI>
__device__ __forceinline__ void layer_epilogue32(const LayerArgs& A, int n, int m0, const float* v) {
    const size_t o = (size_t)n * kH + m0;
    auto ld32 = [](const float* src, float* x) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 a = reinterpret_cast<const float4*>(src)[q];
            x[4 * q] = a.x; x[4 * q + 1] = a.y; x[4 * q + 2] = a.z; x[4 * q + 3] = a.w;
        }
    };
    auto st8 = [](float* dst, const float* x) {
        *reinterpret_cast<float4*>(dst) = make_float4(x[0], x[1], x[2], x[3]);
        *reinterpret_cast<float4*>(dst + 4) = make_float4(x[4], x[5], x[6], x[7]);
    };
    if constexpr (EPI == kFwd) {
#pragma unroll
        for (int j = 0; j < 4; ++j) layer_epilogue8<kFwd>(A, n, m0 + 8 * j, v + 8 * j);  // no loads but the bias
    } else if constexpr (EPI == kBwd) {
        float z[32];
        ld32(A.Z + o, z);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float a[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) a[q] = sigmoid_t(z[8 * j + q]) * v[8 * j + q];
            st8(A.G + o + 8 * j, v + 8 * j);
            st_out8(A, A.outb + o + 8 * j, a, n, m0 + 8 * j, true);
        }
    } else if constexpr (EPI == kFwdT) {
        float z[32];
        ld32(A.Z + o, z);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float a[8], b[8];
            st8(A.Zd + o + 8 * j, v + 8 * j);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float sg = sigmoid_t(z[8 * j + q]);
                a[q] = sg * v[8 * j + q];
                b[q] = A.last ? sg * (1.f - sg) * v[8 * j + q] * A.w5[m0 + 8 * j + q] : 0.f;
            }
            if (A.last) {
                st8(A.outf + o + 8 * j, a);
                st_out8(A, A.outb2 + o + 8 * j, b, n, m0 + 8 * j, true);
            } else {
                st_out8(A, A.outb + o + 8 * j, a, n, m0 + 8 * j, true);
            }
        }
    } else {
        float z[32], zd[32], g[32];
        ld32(A.Z + o, z);
        ld32(A.Zd + o, zd);
        ld32(A.G + o, g);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float a[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = 8 * j + q;
                const float sg = sigmoid_t(z[k]);
                a[q] = sg * v[k] + sg * (1.f - sg) * zd[k] * g[k];
            }
            st_out8(A, A.outb + o + 8 * j, a, n, m0 + 8 * j, true);
        }
    }
}

// One 128-wide layer for the 128 samples n0.. of this CTA: stage the operands that are not in shared
// memory yet (stage_a: the activations from A.in, stage_w: the weights from A.W), issue the MMAs from
// one thread, wait for them (bounded; the MMA barrier completes once per layer, so the layer waits for
// phase `phase`), start fetching the next layer's weights W_next into Bs (free once the MMAs are done),
// run the epilogue from TMEM (which writes the next layer's activations into As when A.smem_next is
// set).  Returns false, with every thread agreeing, when the wait ran out.  On return every thread has
// finished with TMEM and its writes are visible to the CTA.
constexpr int kChainThreads = 256;  // two threads per sample: warps w and w + 4 read the same TMEM lanes

__device__ __forceinline__ void stage_weights(unsigned char* Bs, const __nv_bfloat16* W) {
    for (int c = threadIdx.x; c < 128 * 16; c += kChainThreads) {
        const int r8 = c & 7, q = (c >> 3) & 15, g = c >> 7, r = 8 * g + r8;
        cp_async16_zfill(Bs + g * 2048 + q * 128 + r8 * 16, W + (size_t)r * kH + q * 8, true);
    }
    asm volatile("cp.async.commit_group;\n" ::);
}

template <int EPI>
__device__ bool umma_layer(const LayerArgs& A, int n0, unsigned char* As, unsigned char* Bs, uint32_t tmem,
                           uint64_t* mbar, uint32_t phase, int* s_fail, bool stage_a, bool stage_w,
                           const __nv_bfloat16* W_next) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // staging: consecutive threads fill consecutive 16-byte rows of one core matrix
    if (stage_a) {
        for (int c = tid; c < 128 * 16; c += kChainThreads) {
            const int r8 = c & 7, q = (c >> 3) & 15, g = c >> 7, r = 8 * g + r8;
            const bool valid = n0 + r < A.n;
            cp_async16_zfill(As + g * 2048 + q * 128 + r8 * 16, A.in + (size_t)(valid ? n0 + r : 0) * kH + q * 8,
                             valid);
        }
        asm volatile("cp.async.commit_group;\n" ::);
    }
    if (stage_w) stage_weights(Bs, A.W);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");  // also the weights prefetched by the previous layer
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // generic-proxy writes -> tensor core reads
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (tid == 0) {
        const uint32_t a0 = smem_addr(As), b0 = smem_addr(Bs);
#pragma unroll
        for (int s = 0; s < kH / 16; ++s) {  // K = 16 per instruction: two 128-byte K chunks
            const uint64_t ad = umma_desc(a0 + 256 * s), bd = umma_desc(b0 + 256 * s);
            const uint32_t acc = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                ::"r"(tmem), "l"(ad), "l"(bd), "r"(kUmmaIdesc), "r"(acc));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                     ::"r"(smem_addr(mbar)) : "memory");
    }
    {  // wait for the MMAs, bounded
        unsigned long long t0;
        asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t0));
        uint32_t done = 0;
        while (!done) {
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done) : "r"(smem_addr(mbar)), "r"(phase) : "memory");
            if (!done) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
                if (t - t0 > kUmmaWaitNs) {
                    atomicOr(s_fail, 1);
                    break;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (*reinterpret_cast<volatile int*>(s_fail)) return false;
    if (W_next) stage_weights(Bs, W_next);  // the MMAs have read Bs: fetch the next weights during the epilogue
    // TMEM lane = sample row: warp w reads lanes 32 (w & 3) .. + 31 (its lane quadrant), columns
    // 64 (w >> 2) .. + 63 (its half of the outputs)
    const int quad = warp & 3, half = warp >> 2;
    const int n = n0 + 32 * quad + lane;
#pragma unroll 1
    for (int c = 2 * half; c < 2 * half + 2; ++c) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(32 * quad) << 16) + 32 * c;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (n < A.n) {
            float v[32];
#pragma unroll
            for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
            layer_epilogue32<EPI>(A, n, 32 * c, v);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();  // TMEM read out and the epilogue's global writes done before the next layer
    return true;
}

// TMEM columns and the MMA barrier of a CTA running umma_layer: set up / released by warp 0 and
// thread 0 (the caller syncs after setup).
__device__ void umma_setup(uint32_t* tmem_base, uint64_t* mbar, int* s_fail) {
    const int tid = threadIdx.x;
    if ((tid >> 5) == 0) {  // 128 TMEM columns of 32-bit accumulators for the 128 outputs
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;\n" ::"r"(smem_addr(tmem_base)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        *s_fail = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_addr(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::);
    }
}
__device__ void umma_release(uint32_t tmem) {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;\n" ::"r"(tmem));
    }
}

// ---------------------------------------------------------------------------------------------
// Stress seed: delta_1 = sigma(z1) G_1 (FP32), g = W1^T delta_1 (FP32 master W1), residuals,
// loss and u = dL/dg (rounded into the padded BF16 tangent input).
// ---------------------------------------------------------------------------------------------
__global__ void seed_kernel(int n, const float* theta, const float* Z0, const float* G0, const float* T,
                            const float* w6, const float* sw, float inv_n, __nv_bfloat16* U0, double* loss) {
    __shared__ float W1s[kIn * kH];  // transposed: [k][m]
    __shared__ double red[8];
    for (int i = threadIdx.x; i < kIn * kH; i += blockDim.x) {
        const int m = i / kIn, k = i - m * kIn;
        W1s[k * kH + m] = theta[oW1 + i];
    }
    __syncthreads();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double part = 0.0;
    if (s < n) {
        const float ws = sw[s];  // per-sample weight
        float gk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        for (int m = 0; m < kH; ++m) {
            const float d = sigmoid_t(Z0[(size_t)s * kH + m]) * G0[(size_t)s * kH + m];
#pragma unroll
            for (int k = 0; k < 6; ++k) gk[k] += W1s[k * kH + m] * d;
        }
#pragma unroll
        for (int k = 0; k < kInPad; ++k) {
            float u = 0.f;
            if (k < 6) {
                const float r = gk[k] - T[(size_t)s * 6 + k];
                part += (double)ws * w6[k] * r * r;
                u = 2.f * ws * w6[k] * r * inv_n;
            }
            U0[(size_t)s * kInPad + k] = __float2bfloat16_rn(u);
        }
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += red[w];
        atomicAdd(loss, tot * inv_n);
    }
}

// ---------------------------------------------------------------------------------------------
// The per-sample part of one gradient evaluation in one launch (tcgen05 path).  CTA = 128 threads
// = 128 samples; everything up to the weight gradients is per sample, so a CTA runs it for its own
// samples without waiting for any other CTA: forward primal, backward primal, stress seed, forward
// tangent, backward tangent.  Layer 1 (7 inputs padded to 16) runs on the CUDA cores from the same
// BF16 operands the tensor cores would read (products exact in FP32, FP32 sums); the twelve 128-wide
// layers run as umma_layer, each reusing the CTA's TMEM columns and MMA barrier.  Intermediates go
// to the same global arrays as the per-layer launches of the mma.sync path (the weight-gradient
// kernels read them afterwards, and later layers of this CTA read them back through L2).
// ---------------------------------------------------------------------------------------------
struct ChainArgs {
    int n;
    size_t BH;                              // stride of the per-layer activation arrays (cap x 128)
    const float* theta;                     // FP32 master parameters (biases, w5, W1 for the seed)
    const __nv_bfloat16 *X0, *Wb1, *Wb, *WbT;
    float *Z, *Zd, *G, *Hd4;
    __nv_bfloat16 *Hb, *Hd, *Db, *Ab, *U0;
    const float *T, *w6, *Sw;
    float inv_n;
    double* loss;
};

// Layer 1 for sample s: out[m] = sum_k W1b[m][k] in[s][k] (BF16 values, FP32 arithmetic), then the
// pass's epilogue on 8 outputs at a time.
template <int EPI>
__device__ void layer1_sample(const LayerArgs& A, const float* W1f, int s, int m_begin, int m_end) {
    if (s >= A.n) return;
    float x[kInPad];
    const uint4* src = reinterpret_cast<const uint4*>(A.in + (size_t)s * kInPad);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint4 u = src[h];
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            x[8 * h + 2 * q] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w[q] & 0xffffu)));
            x[8 * h + 2 * q + 1] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w[q] >> 16)));
        }
    }
#pragma unroll 1
    for (int m0 = m_begin; m0 < m_end; m0 += 8) {
        float v[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            float acc = 0.f;
#pragma unroll
            for (int k = 0; k < kInPad; ++k) acc = fmaf(W1f[(m0 + j) * kInPad + k], x[k], acc);
            v[j] = acc;
        }
        layer_epilogue8<EPI>(A, s, m0, v);
    }
}

// Stress seed of sample s (seed_kernel's arithmetic): g = W1^T (sigma(z1) G_1) in FP32, residuals
// against the targets, u = dL/dg into the padded BF16 tangent input; returns the sample's loss term.
__device__ double seed_sample(const ChainArgs& C, const float* W1m, int s) {
    if (s >= C.n) return 0.0;
    const float ws = C.Sw[s];
    float gk[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float* z0 = C.Z + (size_t)s * kH;
    const float* g0 = C.G + (size_t)s * kH;
    for (int m = 0; m < kH; ++m) {
        const float d = sigmoid_t(z0[m]) * g0[m];
#pragma unroll
        for (int k = 0; k < 6; ++k) gk[k] += W1m[k * kH + m] * d;
    }
    double part = 0.0;
#pragma unroll
    for (int k = 0; k < kInPad; ++k) {
        float u = 0.f;
        if (k < 6) {
            const float r = gk[k] - C.T[(size_t)s * 6 + k];
            part += (double)ws * C.w6[k] * r * r;
            u = 2.f * ws * C.w6[k] * r * C.inv_n;
        }
        C.U0[(size_t)s * kInPad + k] = __float2bfloat16_rn(u);
    }
    return part;
}

__global__ void __launch_bounds__(kChainThreads, 1) grad_chain_kernel(ChainArgs C, int* err) {
    extern __shared__ __align__(1024) unsigned char sm_raw[];
    unsigned char* As = sm_raw;                 // activations operand
    unsigned char* Bs = sm_raw + kUmmaOpBytes;  // weights operand
    __shared__ float W1f[kH * kInPad];          // BF16 W1 (padded to 16 inputs) as floats, [m][k]
    __shared__ float W1m[6 * kH];               // FP32 master W1 of the stress inputs, [k][m]
    __shared__ double red[kChainThreads / 32];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;
    // thread t: sample n0 + (t & 127), output half t >> 7 (layer 1); the seed runs on t < 128
    const int tid = threadIdx.x, n0 = blockIdx.x * kUmmaRows, s = n0 + (tid & 127);
    const int m_begin = (tid >> 7) * (kH / 2), m_end = m_begin + kH / 2;
    umma_setup(&tmem_base, &mbar, &s_fail);
    for (int i = tid; i < kH * kInPad; i += kChainThreads) W1f[i] = __bfloat162float(C.Wb1[i]);
    for (int i = tid; i < kH * kIn; i += kChainThreads) {
        const int m = i / kIn, k = i - m * kIn;
        if (k < 6) W1m[k * kH + m] = C.theta[oW1 + i];
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_base;
    uint32_t phase = 0;
    bool ok = true;
    LayerArgs L{};
    L.n = C.n;
    L.w5 = C.theta + oW5;
    L.smem_next = As;  // every epilogue (and layer 1) leaves its output in As as the next layer's operand
    L.n0 = n0;
    // the weights of the 12 tensor-core layers in order; layer k fetches those of layer k + 1 into Bs
    // while its epilogue runs, so only the first layer stages weights itself and no layer stages
    // activations
    auto W_of = [&](int k) -> const __nv_bfloat16* {
        if (k >= 12) return nullptr;
        const int q = k % 6;  // 0..2: W2..W4 (forward), 3..5: transposed W4..W2 (backward)
        return q < 3 ? C.Wb + (size_t)q * kH * kH : C.WbT + (size_t)(5 - q) * kH * kH;
    };
    int k = 0;
    // forward primal
    L.in = C.X0;
    L.bias = C.theta + layer_b(0);
    L.Z = C.Z;
    L.outb = C.Hb;
    L.last = 0;
    layer1_sample<kFwd>(L, W1f, s, m_begin, m_end);
    __syncthreads();
    for (int l = 1; l < 4 && ok; ++l, phase ^= 1) {
        L.W = C.Wb + (size_t)(l - 1) * kH * kH;
        L.in = C.Hb + (l - 1) * C.BH;
        L.bias = C.theta + layer_b(l);
        L.Z = C.Z + l * C.BH;
        L.outb = C.Hb + l * C.BH;
        L.outb2 = C.Db + 3 * C.BH;
        L.last = l == 3;
        ok = umma_layer<kFwd>(L, n0, As, Bs, tmem, &mbar, phase, &s_fail, false, k == 0, W_of(k + 1));
        ++k;
    }
    // backward primal: G_l = W_{l+1}^T delta_{l+1}, delta_l
    for (int l = 2; l >= 0 && ok; --l, phase ^= 1) {
        L.W = C.WbT + (size_t)l * kH * kH;
        L.in = C.Db + (l + 1) * C.BH;
        L.Z = C.Z + l * C.BH;
        L.G = C.G + l * C.BH;
        L.outb = C.Db + l * C.BH;
        L.last = 0;
        ok = umma_layer<kBwd>(L, n0, As, Bs, tmem, &mbar, phase, &s_fail, false, k == 0, W_of(k + 1));
        ++k;
    }
    if (ok) {
        double part = tid < 128 ? seed_sample(C, W1m, s) : 0.0;
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        if (tid == 0) {
            double tot = 0.0;
            for (int w = 0; w < kChainThreads / 32; ++w) tot += red[w];
            atomicAdd(C.loss, tot * C.inv_n);
        }
        // forward tangent along u
        L.in = C.U0;
        L.Z = C.Z;
        L.Zd = C.Zd;
        L.outb = C.Hd;
        L.outb2 = C.Ab + 3 * C.BH;
        L.outf = C.Hd4;
        L.last = 0;
        layer1_sample<kFwdT>(L, W1f, s, m_begin, m_end);
        __syncthreads();
    }
    for (int l = 1; l < 4 && ok; ++l, phase ^= 1) {
        L.W = C.Wb + (size_t)(l - 1) * kH * kH;
        L.in = C.Hd + (l - 1) * C.BH;
        L.Z = C.Z + l * C.BH;
        L.Zd = C.Zd + l * C.BH;
        L.outb = C.Hd + l * C.BH;
        L.outb2 = C.Ab + 3 * C.BH;
        L.outf = C.Hd4;
        L.last = l == 3;
        ok = umma_layer<kFwdT>(L, n0, As, Bs, tmem, &mbar, phase, &s_fail, false, k == 0, W_of(k + 1));
        ++k;
    }
    // backward tangent: a_l from W_{l+1}^T a_{l+1}
    for (int l = 2; l >= 0 && ok; --l, phase ^= 1) {
        L.W = C.WbT + (size_t)l * kH * kH;
        L.in = C.Ab + (l + 1) * C.BH;
        L.Z = C.Z + l * C.BH;
        L.Zd = C.Zd + l * C.BH;
        L.G = C.G + l * C.BH;
        L.outb = C.Ab + l * C.BH;
        L.last = 0;
        ok = umma_layer<kBwdT>(L, n0, As, Bs, tmem, &mbar, phase, &s_fail, false, k == 0, W_of(k + 1));
        ++k;
    }
    if (!ok && tid == 0) atomicOr(err, 1);
    umma_release(tmem);
}

// ---------------------------------------------------------------------------------------------
// Weight gradients: dW[m][k] += sum_n A[n][m] P[n][k] + D[n][m] Q[n][k] over a chunk of samples.
// CTA = 8 warps, warp w owns rows [16w, 16w+16) x all NK columns.
// ---------------------------------------------------------------------------------------------
struct GradArgs {
    int n;
    const __nv_bfloat16* A[4];   // a_l      [n][128]
    const __nv_bfloat16* D[4];   // delta_l  [n][128]
    const __nv_bfloat16* P[4];   // h_{l-1}  [n][NK]
    const __nv_bfloat16* Q[4];   // hdot_{l-1}
    float* dW[4];                // [128][NK] (layer 0: [128][7] written from a [128][16] tile)
};

template <int NK>
__global__ void __launch_bounds__(256) weight_grad_kernel(GradArgs G, int layer0) {
    constexpr int LDA = kH + 8, LDP = NK + 8, SUB = 32;
    __shared__ __align__(16) __nv_bfloat16 As[SUB * LDA];
    __shared__ __align__(16) __nv_bfloat16 Ds[SUB * LDA];
    __shared__ __align__(16) __nv_bfloat16 Ps[SUB * LDP];
    __shared__ __align__(16) __nv_bfloat16 Qs[SUB * LDP];
    const int layer = layer0 + blockIdx.y;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    constexpr int NT = NK / 8;
    float acc[NT][4];
#pragma unroll
    for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[j][k] = 0.f;
    const int c0 = blockIdx.x * kChunk;
    for (int s0 = c0; s0 < min(G.n, c0 + kChunk); s0 += SUB) {
        __syncthreads();
        for (int c = tid; c < SUB * (kH / 8); c += 256) {
            const int r = c / (kH / 8), q = c - r * (kH / 8);
            uint4 va = make_uint4(0, 0, 0, 0), vd = va;
            if (s0 + r < G.n) {
                va = *reinterpret_cast<const uint4*>(G.A[layer] + (size_t)(s0 + r) * kH + q * 8);
                vd = *reinterpret_cast<const uint4*>(G.D[layer] + (size_t)(s0 + r) * kH + q * 8);
            }
            *reinterpret_cast<uint4*>(As + r * LDA + q * 8) = va;
            *reinterpret_cast<uint4*>(Ds + r * LDA + q * 8) = vd;
        }
        for (int c = tid; c < SUB * (NK / 8); c += 256) {
            const int r = c / (NK / 8), q = c - r * (NK / 8);
            uint4 vp = make_uint4(0, 0, 0, 0), vq = vp;
            if (s0 + r < G.n) {
                vp = *reinterpret_cast<const uint4*>(G.P[layer] + (size_t)(s0 + r) * NK + q * 8);
                vq = *reinterpret_cast<const uint4*>(G.Q[layer] + (size_t)(s0 + r) * NK + q * 8);
            }
            *reinterpret_cast<uint4*>(Ps + r * LDP + q * 8) = vp;
            *reinterpret_cast<uint4*>(Qs + r * LDP + q * 8) = vq;
        }
        __syncthreads();
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
            const __nv_bfloat16* L = pass ? Ds : As;
            const __nv_bfloat16* R = pass ? Qs : Ps;
#pragma unroll
            for (int k0 = 0; k0 < SUB; k0 += 16) {
                const int m = 16 * warp + g;
                uint32_t af[4];
                af[0] = pack2(L[(k0 + 2 * t) * LDA + m], L[(k0 + 2 * t + 1) * LDA + m]);
                af[1] = pack2(L[(k0 + 2 * t) * LDA + m + 8], L[(k0 + 2 * t + 1) * LDA + m + 8]);
                af[2] = pack2(L[(k0 + 2 * t + 8) * LDA + m], L[(k0 + 2 * t + 9) * LDA + m]);
                af[3] = pack2(L[(k0 + 2 * t + 8) * LDA + m + 8], L[(k0 + 2 * t + 9) * LDA + m + 8]);
#pragma unroll
                for (int nt = 0; nt < NT; ++nt) {
                    uint32_t bf[2];
                    bf[0] = pack2(R[(k0 + 2 * t) * LDP + 8 * nt + g], R[(k0 + 2 * t + 1) * LDP + 8 * nt + g]);
                    bf[1] = pack2(R[(k0 + 2 * t + 8) * LDP + 8 * nt + g], R[(k0 + 2 * t + 9) * LDP + 8 * nt + g]);
                    mma_bf16(acc[nt], af, bf);
                }
            }
        }
    }
    float* dW = G.dW[layer];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int m = 16 * warp + g + 8 * (q >> 1), k = 8 * nt + 2 * t + (q & 1);
            if (NK == kH) atomicAdd(dW + m * kH + k, acc[nt][q]);
            else if (k < kIn) atomicAdd(dW + m * kIn + k, acc[nt][q]);
        }
}

// bias gradients (sums of a_l) and dw5 (sum of hdot_4): thread = feature, CTA = sample chunk
__global__ void bias_grad_kernel(int n, const __nv_bfloat16* const* A, const float* Hd4, float* grad) {
    const int m = threadIdx.x;
    const int s0 = blockIdx.x * kChunk, s1 = min(n, s0 + kChunk);
    float b[4] = {0.f, 0.f, 0.f, 0.f}, w = 0.f;
    for (int s = s0; s < s1; ++s) {
#pragma unroll
        for (int l = 0; l < 4; ++l) b[l] += __bfloat162float(A[l][(size_t)s * kH + m]);
        w += Hd4[(size_t)s * kH + m];
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) atomicAdd(grad + layer_b(l) + m, b[l]);
    atomicAdd(grad + oW5 + m, w);
}

// Step bookkeeping inside the captured training step: ctr[0] = Adam step t (incremented),
// ctr[1] = offset of the batch in the epoch permutation; hp = [lr, 1/(1-beta1^t), 1/(1-beta2^t)]
// with lr = lr0 * decay^(t-1).
__global__ void step_kernel(int* ctr, float lr0, float decay, float b1, float b2, float* hp) {
    const int t = ++ctr[0];
    hp[0] = lr0 * powf(decay, (float)(t - 1));
    hp[1] = 1.f / (1.f - powf(b1, (float)t));
    hp[2] = 1.f / (1.f - powf(b2, (float)t));
}
__global__ void gather_rows_kernel(int nb, int* ctr, const int* idx, const float* Xall, const float* Tall,
                                   const float* Swall, float* X, float* T, float* Sw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const int r = idx[ctr[1] + i];
    for (int k = 0; k < kIn; ++k) X[(size_t)i * kIn + k] = Xall[(size_t)r * kIn + k];
    for (int k = 0; k < 6; ++k) T[(size_t)i * 6 + k] = Tall[(size_t)r * 6 + k];
    Sw[i] = Swall[r];
}
__global__ void advance_kernel(int* ctr, int nb) { ctr[1] += nb; }

// Adam on the FP32 master vector; grad re-zeroed; BF16 copies (and transposes) refreshed.
__global__ void adam_kernel(float* theta, float* grad, float* m1, float* m2, const float* hp, float b1, float b2,
                            float eps, __nv_bfloat16* Wb1, __nv_bfloat16* Wb, __nv_bfloat16* WbT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kNParams) return;
    const float gr = grad[i];
    grad[i] = 0.f;
    const float a = b1 * m1[i] + (1.f - b1) * gr, v = b2 * m2[i] + (1.f - b2) * gr * gr;
    m1[i] = a;
    m2[i] = v;
    const float th = theta[i] - hp[0] * (a * hp[1]) / (sqrtf(v * hp[2]) + eps);
    theta[i] = th;
    const __nv_bfloat16 hb = __float2bfloat16_rn(th);
    if (i < oB1) {
        const int m = i / kIn, k = i - m * kIn;
        Wb1[m * kInPad + k] = hb;
    } else {
        for (int l = 1; l < 4; ++l) {
            const int o = layer_w(l);
            if (i >= o && i < o + kH * kH) {
                const int m = (i - o) / kH, k = (i - o) % kH;
                Wb[(size_t)(l - 1) * kH * kH + m * kH + k] = hb;
                WbT[(size_t)(l - 1) * kH * kH + k * kH + m] = hb;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Inference: per point, S (6) and the material tangent (36), pushed forward with F to the
// Cauchy stress and spatial tangent (element-loop external material layout), plus a range flag.
// CTA = 256 threads, 16 points; thread (m = tid % 128, half = tid / 128) owns points 8 half..+8.
// ---------------------------------------------------------------------------------------------
constexpr int kTP = 16;
struct InferArgs {
    int n;                       // points
    const double* F;             // [9][ldF] row-major F per point (FP64) or nullptr
    long long ldF;
    const double* C6;            // [n][6] right Cauchy-Green (used when F == nullptr)
    const double* vf;            // per point, indexed vf[q % vf_mod]
    int vf_mod;
    const float* theta;          // master parameters
    const float* WT;             // [3][128][128] transposed W2..W4 (FP32)
    float sC, sW, vf0, svf;
    const float* lo;             // [7] training box of x
    const float* hi;
    double* S;                   // [n][6] (nullable)
    double* Cm;                  // [n][36] (nullable)
    int* flag;                   // [n] 1 = outside the training box (nullable)
    // external-material output: state[(v*8 + gp)*ld + e] for point q = gp*n_elem + e
    void* state;
    int state_f32;
    long long ld;
    int n_elem;
    // reference-state correction: S(C = I, vf) tabulated over [tab_lo, tab_hi] (n_tab rows of 6),
    // subtracted from every stress so that the undeformed state is stress-free (nullable)
    const double* s0tab;
    int n_tab;
    double tab_lo, tab_hi;
};

__global__ void __launch_bounds__(256) infer_kernel(InferArgs A) {
    extern __shared__ __align__(16) float sm[];
    float* Zs = sm;                        // [4][kTP][128]
    float* Cs = Zs + 4 * kTP * kH;         // [4][kTP][128]  G_l sigma'(z_l)
    float* Hb = Cs + 4 * kTP * kH;         // [kTP][128] activation / adjoint work vector
    float* Jin = Hb + kTP * kH;            // [kTP][128][8]  (6 used)
    float* Jout = Jin + kTP * kH * 8;      // [kTP][128][8]
    float* Xs = Jout + kTP * kH * 8;       // [kTP][8]
    float* Hs = Xs + kTP * 8;              // [kTP][6][6] Hessian accumulators
    float* Gs = Hs + kTP * 36;             // [kTP][8] de/dx
    const float* th = A.theta;
    const int tid = threadIdx.x, m = tid & (kH - 1), half = tid >> 7;
    const int ntiles = (A.n + kTP - 1) / kTP;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int q0 = tile * kTP;
        __syncthreads();
        if (tid < kTP) {
            const int q = q0 + tid;
            float x[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (q < A.n) {
                double C[6];
                if (A.F) {
                    double F[9];
                    for (int k = 0; k < 9; ++k) F[k] = A.F[k * A.ldF + q];
                    for (int p = 0; p < 6; ++p) {
                        const int I = p < 3 ? p : (p == 3 ? 0 : (p == 4 ? 1 : 0));
                        const int J = p < 3 ? p : (p == 3 ? 1 : 2);
                        C[p] = F[I] * F[J] + F[3 + I] * F[3 + J] + F[6 + I] * F[6 + J];
                    }
                } else {
                    for (int p = 0; p < 6; ++p) C[p] = A.C6[(size_t)q * 6 + p];
                }
                for (int p = 0; p < 6; ++p) x[p] = (float)((C[p] - (p < 3 ? 1.0 : 0.0)) / A.sC);
                x[6] = (float)((A.vf[q % A.vf_mod] - A.vf0) / A.svf);
                if (A.flag) {
                    int out = 0;
                    for (int k = 0; k < kIn; ++k) out |= (x[k] < A.lo[k] || x[k] > A.hi[k]) ? 1 : 0;
                    A.flag[q] = out;
                }
            }
            for (int k = 0; k < 8; ++k) Xs[tid * 8 + k] = x[k];
        }
        for (int i = tid; i < kTP * 36; i += 256) Hs[i] = 0.f;
        __syncthreads();
        // ---- pass 1: forward primal (thread: unit m, points half*8 .. +8) ----
        {
            float acc[8];
            const float b = th[oB1 + m];
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                float z = b;
#pragma unroll
                for (int k = 0; k < kIn; ++k) z += th[oW1 + m * kIn + k] * Xs[(half * 8 + p) * 8 + k];
                acc[p] = z;
            }
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                Zs[(0 * kTP + half * 8 + p) * kH + m] = acc[p];
                Hb[(half * 8 + p) * kH + m] = softplus_f(acc[p]);
            }
        }
        for (int l = 1; l < 4; ++l) {
            __syncthreads();
            float acc[8];
            const float* W = th + layer_w(l) + m * kH;
#pragma unroll
            for (int p = 0; p < 8; ++p) acc[p] = th[layer_b(l) + m];
            for (int i = 0; i < kH; i += 4) {
                const float4 w = *reinterpret_cast<const float4*>(W + i);
#pragma unroll
                for (int p = 0; p < 8; ++p) {
                    const float4 h = *reinterpret_cast<const float4*>(Hb + (half * 8 + p) * kH + i);
                    acc[p] += w.x * h.x + w.y * h.y + w.z * h.z + w.w * h.w;
                }
            }
            __syncthreads();
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                Zs[(l * kTP + half * 8 + p) * kH + m] = acc[p];
                Hb[(half * 8 + p) * kH + m] = softplus_f(acc[p]);
            }
        }
        // ---- pass 2: backward; G_4 = w5, delta_l = sigma(z_l) G_l, G_{l-1} = W_l^T delta_l ----
        __syncthreads();
        {
            const float w5 = th[oW5 + m];
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const float z = Zs[(3 * kTP + half * 8 + p) * kH + m];
                const float s = sigmoid_f(z);
                Cs[(3 * kTP + half * 8 + p) * kH + m] = w5 * s * (1.f - s);
                Hb[(half * 8 + p) * kH + m] = s * w5;
            }
        }
        for (int l = 3; l >= 1; --l) {
            __syncthreads();
            float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            const float* WT = A.WT + (size_t)(l - 1) * kH * kH + m * kH;  // row m of W_l^T
            for (int i = 0; i < kH; i += 4) {
                const float4 w = *reinterpret_cast<const float4*>(WT + i);
#pragma unroll
                for (int p = 0; p < 8; ++p) {
                    const float4 d = *reinterpret_cast<const float4*>(Hb + (half * 8 + p) * kH + i);
                    acc[p] += w.x * d.x + w.y * d.y + w.z * d.z + w.w * d.w;
                }
            }
            __syncthreads();
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const float s = sigmoid_f(Zs[((l - 1) * kTP + half * 8 + p) * kH + m]);
                Cs[((l - 1) * kTP + half * 8 + p) * kH + m] = acc[p] * s * (1.f - s);
                Hb[(half * 8 + p) * kH + m] = s * acc[p];
            }
        }
        __syncthreads();
        // de/dx_k = sum_m W1[m][k] delta_1[m]
        if (tid < kTP * 6) {
            const int p = tid / 6, k = tid - 6 * p;
            float s = 0.f;
            for (int mm = 0; mm < kH; ++mm) s += th[oW1 + mm * kIn + k] * Hb[p * kH + mm];
            Gs[p * 8 + k] = s;
        }
        // ---- pass 3: Jacobians J_l = dz_l/dx (first 6 inputs), Hessian accumulation ----
        for (int i = tid; i < kTP * kH; i += 256) {
            const int p = i / kH, mm = i - p * kH;
#pragma unroll
            for (int k = 0; k < 6; ++k) Jin[(p * kH + mm) * 8 + k] = th[oW1 + mm * kIn + k];
        }
        for (int l = 0; l < 4; ++l) {
            __syncthreads();
            // H += J_l^T diag(c_l) J_l: thread = (point, pair) over 16 x 21 pairs
            for (int i = tid; i < kTP * 21; i += 256) {
                const int p = i / 21, r = i - 21 * p;
                int a = 0, rr = r;
                while (rr >= 6 - a) { rr -= 6 - a; ++a; }
                const int b = a + rr;
                float s = 0.f;
                const float* c = Cs + (l * kTP + p) * kH;
                const float* J = Jin + p * kH * 8;
                for (int mm = 0; mm < kH; ++mm) s += J[mm * 8 + a] * c[mm] * J[mm * 8 + b];
                Hs[p * 36 + a * 6 + b] += s;
            }
            if (l == 3) break;
            // Jin <- sigma(z_l) J_l (in place, per element)
            __syncthreads();
            for (int i = tid; i < kTP * kH; i += 256) {
                const int p = i / kH, mm = i - p * kH;
                const float s = sigmoid_f(Zs[(l * kTP + p) * kH + mm]);
#pragma unroll
                for (int k = 0; k < 6; ++k) Jin[(p * kH + mm) * 8 + k] *= s;
            }
            __syncthreads();
            // Jout[p][m][k] = sum_i W_{l+1}[m][i] Jin[p][i][k]
            float acc[8][6];
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int k = 0; k < 6; ++k) acc[p][k] = 0.f;
            const float* W = th + layer_w(l + 1) + m * kH;
            for (int i4 = 0; i4 < kH; i4 += 4) {
                const float4 w4 = *reinterpret_cast<const float4*>(W + i4);
                const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
                for (int ii = 0; ii < 4; ++ii) {
                    const float w = wv[ii];
                    const int i = i4 + ii;
#pragma unroll
                    for (int p = 0; p < 8; ++p) {
                        const float4 j0 = *reinterpret_cast<const float4*>(Jin + ((half * 8 + p) * kH + i) * 8);
                        const float2 j1 = *reinterpret_cast<const float2*>(Jin + ((half * 8 + p) * kH + i) * 8 + 4);
                        acc[p][0] += w * j0.x;
                        acc[p][1] += w * j0.y;
                        acc[p][2] += w * j0.z;
                        acc[p][3] += w * j0.w;
                        acc[p][4] += w * j1.x;
                        acc[p][5] += w * j1.y;
                    }
                }
            }
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int k = 0; k < 6; ++k) Jout[((half * 8 + p) * kH + m) * 8 + k] = acc[p][k];
            __syncthreads();
            float* tmp = Jin;
            Jin = Jout;
            Jout = tmp;
        }
        __syncthreads();
        // ---- outputs: S, material tangent, push-forward ----
        if (tid < kTP) {
            const int q = q0 + tid;
            if (q < A.n) {
                const double av[6] = {2, 2, 2, 1, 1, 1};
                double S[6], Cm[6][6];
                for (int a = 0; a < 6; ++a) S[a] = av[a] * (A.sW / A.sC) * Gs[tid * 8 + a];
                if (A.s0tab) {  // W - S0(vf):(C - I)/2 keeps the energy form and the tangent
                    const double v = A.vf[q % A.vf_mod];
                    double tpos = (v - A.tab_lo) / (A.tab_hi - A.tab_lo) * (A.n_tab - 1);
                    tpos = fmin(fmax(tpos, 0.0), (double)(A.n_tab - 1));
                    const int i0 = min((int)tpos, A.n_tab - 2);
                    const double w = tpos - i0;
                    for (int a = 0; a < 6; ++a) S[a] -= (1.0 - w) * A.s0tab[6 * i0 + a] + w * A.s0tab[6 * (i0 + 1) + a];
                }
                for (int a = 0; a < 6; ++a)
                    for (int b = a; b < 6; ++b) {
                        const double v = av[a] * av[b] * (A.sW / ((double)A.sC * A.sC)) * Hs[tid * 36 + a * 6 + b];
                        Cm[a][b] = v;
                        Cm[b][a] = v;
                    }
                if (A.S)
                    for (int a = 0; a < 6; ++a) A.S[(size_t)q * 6 + a] = S[a];
                if (A.Cm)
                    for (int a = 0; a < 36; ++a) A.Cm[(size_t)q * 36 + a] = Cm[a / 6][a % 6];
                if (A.state && A.F) {
                    double F[9];
                    for (int k = 0; k < 9; ++k) F[k] = A.F[k * A.ldF + q];
                    const double J = F[0] * (F[4] * F[8] - F[5] * F[7]) - F[1] * (F[3] * F[8] - F[5] * F[6]) +
                                     F[2] * (F[3] * F[7] - F[4] * F[6]);
                    const int vi[6] = {0, 1, 2, 0, 1, 0}, vj[6] = {0, 1, 2, 1, 2, 2};
                    // Q[p][r]: Voigt push-forward of a symmetric tensor, shear columns doubled
                    double Q[6][6];
                    for (int p = 0; p < 6; ++p)
                        for (int r = 0; r < 6; ++r) {
                            const int i = vi[p], j = vj[p], I = vi[r], Jx = vj[r];
                            Q[p][r] = F[3 * i + I] * F[3 * j + Jx] + (r >= 3 ? F[3 * i + Jx] * F[3 * j + I] : 0.0);
                        }
                    double sig[6], Dsp[21];
                    for (int p = 0; p < 6; ++p) {
                        double s = 0.0;
                        for (int r = 0; r < 6; ++r) s += Q[p][r] * S[r];
                        sig[p] = s / J;
                    }
                    double QC[6][6];
                    for (int p = 0; p < 6; ++p)
                        for (int s = 0; s < 6; ++s) {
                            double v = 0.0;
                            for (int r = 0; r < 6; ++r) v += Q[p][r] * Cm[r][s];
                            QC[p][s] = v;
                        }
                    int u = 0;
                    for (int p = 0; p < 6; ++p)
                        for (int qq = p; qq < 6; ++qq) {
                            double v = 0.0;
                            for (int s = 0; s < 6; ++s) v += QC[p][s] * Q[qq][s];
                            Dsp[u++] = v / J;
                        }
                    const int gp = q / A.n_elem, e = q - gp * A.n_elem;
                    for (int v = 0; v < 27; ++v) {
                        const double val = v < 6 ? sig[v] : Dsp[v - 6];
                        const size_t o = ((size_t)v * 8 + gp) * A.ld + e;
                        if (A.state_f32) static_cast<float*>(A.state)[o] = (float)val;
                        else static_cast<double*>(A.state)[o] = val;
                    }
                }
            }
        }
    }
}
constexpr size_t kInferSmem = sizeof(float) * (8 * kTP * kH + kTP * kH + 2 * kTP * kH * 8 + kTP * 8 + kTP * 36 + kTP * 8);

// ---------------------------------------------------------------------------------------------
// Handle
// ---------------------------------------------------------------------------------------------
struct Sur {
    int device = 0, cap = 0;
    cudaStream_t stream = nullptr;
    std::string msg;
    float scales[4] = {0.15f, 1.0f, 0.25f, 0.15f};  // s_C, s_W, vf0, s_vf
    float lo[kIn], hi[kIn];
    // parameters
    float *theta = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr, *hp = nullptr, *WT = nullptr;
    float *box = nullptr;  // [14] lo, hi
    double* s0tab = nullptr;  // [kTab][6] reference-state stress over the vf range (when s0_on)
    int s0_on = 0;
    double tab_lo = 0.0, tab_hi = 1.0;
    __nv_bfloat16 *Wb1 = nullptr, *Wb = nullptr, *WbT = nullptr;
    int step = 0;
    // workspace for batches of cap samples
    __nv_bfloat16 *X0 = nullptr, *U0 = nullptr, *Hb = nullptr, *Hd = nullptr, *Db = nullptr, *Ab = nullptr;
    float *Z = nullptr, *Zd = nullptr, *G = nullptr, *Hd4 = nullptr, *T = nullptr, *w6 = nullptr;
    float* Sw = nullptr;  // [cap] per-sample loss weights of the current batch
    __nv_bfloat16** Aptr = nullptr;  // device array of the 4 a_l pointers
    double* loss = nullptr;
    int* ctr = nullptr;  // [2] Adam step, batch offset
    int gemm_path = 1;   // 128-wide layer GEMMs: 1 tcgen05 (TMEM accumulators, default), 0 mma.sync on warps
    int* err = nullptr;  // set by a tensor-core GEMM whose MMA completion wait exceeded its bound
    ~Sur() {
        void* p[] = {theta, grad, m1, m2, hp, WT, box, Wb1, Wb, WbT, X0, U0, Hb, Hd, Db, Ab, Z, Zd, G, Hd4, T, w6, Aptr, loss, ctr, Sw, s0tab, err};
        for (void* q : p)
            if (q) cudaFree(q);
        if (stream) cudaStreamDestroy(stream);
    }
};

#define CKS(call)                                                              \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            s->msg = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return CEOS_E_CUDA;                                                \
        }                                                                      \
    } while (0)

// BF16 copies and FP32 transposes of the weights from the master vector (host-side refresh)
__global__ void refresh_kernel(const float* theta, __nv_bfloat16* Wb1, __nv_bfloat16* Wb, __nv_bfloat16* WbT,
                               float* WT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kH * kInPad) {
        const int m = i / kInPad, k = i - m * kInPad;
        Wb1[i] = __float2bfloat16_rn(k < kIn ? theta[oW1 + m * kIn + k] : 0.f);
    }
    if (i < 3 * kH * kH) {
        const int l = i / (kH * kH), r = i - l * kH * kH, m = r / kH, k = r - m * kH;
        const float v = theta[layer_w(l + 1) + r];
        Wb[i] = __float2bfloat16_rn(v);
        WbT[(size_t)l * kH * kH + k * kH + m] = __float2bfloat16_rn(v);
        WT[(size_t)l * kH * kH + k * kH + m] = v;
    }
}
__global__ void transpose_f32_kernel(const float* theta, float* WT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * kH * kH) {
        const int l = i / (kH * kH), r = i - l * kH * kH, m = r / kH, k = r - m * kH;
        WT[(size_t)l * kH * kH + k * kH + m] = theta[layer_w(l + 1) + r];
    }
}
__global__ void pack_inputs_kernel(int n, const float* X, __nv_bfloat16* X0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * kInPad) return;
    const int s = i / kInPad, k = i - s * kInPad;
    X0[i] = __float2bfloat16_rn(k < kIn ? X[(size_t)s * kIn + k] : 0.f);
}

// One 128-wide layer GEMM (K = 128) of the mma.sync path.
template <int EPI>
void launch_layer(Sur* s, const LayerArgs& L, int n, cudaStream_t st) {
    layer_gemm_kernel<kH, EPI><<<(n + kTileN - 1) / kTileN, 128, 0, st>>>(L);
}

int weight_grads(Sur* s, int n, cudaStream_t st);

// One gradient evaluation over n <= cap samples already on the device (X [n][7], T [n][6]):
// accumulates dL/dtheta into s->grad and the loss into s->loss.
int grad_device(Sur* s, int n, const float* dX) {
    cudaStream_t st = s->stream;
    const size_t BH = (size_t)s->cap * kH;
    pack_inputs_kernel<<<(n * kInPad + 255) / 256, 256, 0, st>>>(n, dX, s->X0);
    if (s->gemm_path == 1) {  // tcgen05: the per-sample chain in one launch, then the weight gradients
        ChainArgs C{};
        C.n = n;
        C.BH = BH;
        C.theta = s->theta;
        C.X0 = s->X0;
        C.Wb1 = s->Wb1;
        C.Wb = s->Wb;
        C.WbT = s->WbT;
        C.Z = s->Z;
        C.Zd = s->Zd;
        C.G = s->G;
        C.Hd4 = s->Hd4;
        C.Hb = s->Hb;
        C.Hd = s->Hd;
        C.Db = s->Db;
        C.Ab = s->Ab;
        C.U0 = s->U0;
        C.T = s->T;
        C.w6 = s->w6;
        C.Sw = s->Sw;
        C.inv_n = 1.f / n;
        C.loss = s->loss;
        grad_chain_kernel<<<(n + kUmmaRows - 1) / kUmmaRows, kChainThreads, 2 * kUmmaOpBytes, st>>>(C, s->err);
        return weight_grads(s, n, st);
    }
    const int nb = (n + kTileN - 1) / kTileN;
    LayerArgs L{};
    L.n = n;
    L.w5 = s->theta + oW5;
    // forward primal
    for (int l = 0; l < 4; ++l) {
        L.bias = s->theta + layer_b(l);
        L.Z = s->Z + l * BH;
        L.outb = s->Hb + l * BH;
        L.outb2 = s->Db + 3 * BH;
        L.last = l == 3;
        if (l == 0) {
            L.W = s->Wb1;
            L.in = s->X0;
            layer_gemm_kernel<kInPad, kFwd><<<nb, 128, 0, st>>>(L);
        } else {
            L.W = s->Wb + (size_t)(l - 1) * kH * kH;
            L.in = s->Hb + (l - 1) * BH;
            launch_layer<kFwd>(s, L, n, st);
        }
    }
    // backward primal: G_{l} = W_{l+1}^T delta_{l+1}, delta_l
    for (int l = 2; l >= 0; --l) {
        L.W = s->WbT + (size_t)l * kH * kH;   // transposed W_{l+2} (1-based) = layer index l+1
        L.in = s->Db + (l + 1) * BH;
        L.Z = s->Z + l * BH;
        L.G = s->G + l * BH;
        L.outb = s->Db + l * BH;
        L.last = 0;
        launch_layer<kBwd>(s, L, n, st);
    }
    seed_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, s->theta, s->Z, s->G, s->T, s->w6, s->Sw, 1.f / n, s->U0,
                                                 s->loss);
    // forward tangent
    for (int l = 0; l < 4; ++l) {
        L.Z = s->Z + l * BH;
        L.Zd = s->Zd + l * BH;
        L.outb = s->Hd + l * BH;
        L.outb2 = s->Ab + 3 * BH;
        L.outf = s->Hd4;
        L.last = l == 3;
        if (l == 0) {
            L.W = s->Wb1;
            L.in = s->U0;
            layer_gemm_kernel<kInPad, kFwdT><<<nb, 128, 0, st>>>(L);
        } else {
            L.W = s->Wb + (size_t)(l - 1) * kH * kH;
            L.in = s->Hd + (l - 1) * BH;
            launch_layer<kFwdT>(s, L, n, st);
        }
    }
    // backward tangent: a_l from W_{l+1}^T a_{l+1}
    for (int l = 2; l >= 0; --l) {
        L.W = s->WbT + (size_t)l * kH * kH;
        L.in = s->Ab + (l + 1) * BH;
        L.Z = s->Z + l * BH;
        L.Zd = s->Zd + l * BH;
        L.G = s->G + l * BH;
        L.outb = s->Ab + l * BH;
        L.last = 0;
        launch_layer<kBwdT>(s, L, n, st);
    }
    return weight_grads(s, n, st);
}

// dW_l = a_l h_{l-1}^T + delta_l hdot_{l-1}^T and the bias gradients, over all n samples.
int weight_grads(Sur* s, int n, cudaStream_t st) {
    const size_t BH = (size_t)s->cap * kH;
    GradArgs G{};
    G.n = n;
    for (int l = 0; l < 4; ++l) {
        G.A[l] = s->Ab + l * BH;
        G.D[l] = s->Db + l * BH;
        G.P[l] = l == 0 ? s->X0 : s->Hb + (l - 1) * BH;
        G.Q[l] = l == 0 ? s->U0 : s->Hd + (l - 1) * BH;
        G.dW[l] = s->grad + layer_w(l);
    }
    const int nc = (n + kChunk - 1) / kChunk;
    weight_grad_kernel<kInPad><<<dim3(nc, 1), 256, 0, st>>>(G, 0);
    weight_grad_kernel<kH><<<dim3(nc, 3), 256, 0, st>>>(G, 1);
    bias_grad_kernel<<<nc, kH, 0, st>>>(n, s->Aptr, s->Hd4, s->grad);
    CKS(cudaGetLastError());
    return 0;
}

int refresh(Sur* s) {
    refresh_kernel<<<(3 * kH * kH + 255) / 256, 256, 0, s->stream>>>(s->theta, s->Wb1, s->Wb, s->WbT, s->WT);
    CKS(cudaGetLastError());
    return 0;
}

}  // namespace

// -------------------------------------------------------------------------------------------------
extern "C" int ceos_sur_create(int batch_max, int device, void** handle) {
    if (batch_max < 1 || !handle) return CEOS_E_ARG;
    *handle = nullptr;
    Sur* s = new Sur();
    s->device = device;
    s->cap = (batch_max + kChunk - 1) / kChunk * kChunk;
    for (int k = 0; k < kIn; ++k) { s->lo[k] = -1.f; s->hi[k] = 1.f; }
    if (cudaSetDevice(device) != cudaSuccess) { delete s; return CEOS_E_CUDA; }
    const size_t BH = (size_t)s->cap * kH;
    bool ok = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) == cudaSuccess;
    auto al = [&](void** p, size_t bytes) {
        if (ok) ok = cudaMalloc(p, bytes) == cudaSuccess && cudaMemset(*p, 0, bytes) == cudaSuccess;
    };
    al((void**)&s->theta, sizeof(float) * kNParams);
    al((void**)&s->grad, sizeof(float) * kNParams);
    al((void**)&s->m1, sizeof(float) * kNParams);
    al((void**)&s->m2, sizeof(float) * kNParams);
    al((void**)&s->hp, sizeof(float) * 4);
    al((void**)&s->WT, sizeof(float) * 3 * kH * kH);
    al((void**)&s->box, sizeof(float) * 2 * kIn);
    al((void**)&s->Wb1, sizeof(__nv_bfloat16) * kH * kInPad);
    al((void**)&s->Wb, sizeof(__nv_bfloat16) * 3 * kH * kH);
    al((void**)&s->WbT, sizeof(__nv_bfloat16) * 3 * kH * kH);
    al((void**)&s->X0, sizeof(__nv_bfloat16) * s->cap * kInPad);
    al((void**)&s->U0, sizeof(__nv_bfloat16) * s->cap * kInPad);
    al((void**)&s->Hb, sizeof(__nv_bfloat16) * 4 * BH);
    al((void**)&s->Hd, sizeof(__nv_bfloat16) * 4 * BH);
    al((void**)&s->Db, sizeof(__nv_bfloat16) * 4 * BH);
    al((void**)&s->Ab, sizeof(__nv_bfloat16) * 4 * BH);
    al((void**)&s->Z, sizeof(float) * 4 * BH);
    al((void**)&s->Zd, sizeof(float) * 4 * BH);
    al((void**)&s->G, sizeof(float) * 4 * BH);
    al((void**)&s->Hd4, sizeof(float) * BH);
    al((void**)&s->T, sizeof(float) * 6 * (size_t)s->cap);
    al((void**)&s->Sw, sizeof(float) * (size_t)s->cap);
    al((void**)&s->w6, sizeof(float) * 6);
    al((void**)&s->Aptr, sizeof(void*) * 4);
    al((void**)&s->loss, sizeof(double));
    al((void**)&s->ctr, sizeof(int) * 2);
    al((void**)&s->err, sizeof(int));
    if (ok)
        ok = cudaFuncSetAttribute(grad_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kUmmaOpBytes) ==
             cudaSuccess;
    if (ok) {
        __nv_bfloat16* ap[4] = {s->Ab, s->Ab + BH, s->Ab + 2 * BH, s->Ab + 3 * BH};
        ok = cudaMemcpy(s->Aptr, ap, sizeof(ap), cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (!ok) { delete s; return CEOS_E_CUDA; }
    *handle = s;
    return 0;
}

extern "C" int ceos_sur_n_params(void) { return kNParams; }

namespace {
// A tensor-core layer GEMM whose MMA completion wait gave up leaves its outputs unwritten.
int gemm_error(Sur* s) {
    int e = 0;
    CKS(cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!e) return 0;
    CKS(cudaMemset(s->err, 0, sizeof(int)));
    s->msg = "tensor-core layer GEMM: the MMA completion wait exceeded its bound";
    return CEOS_E_CUDA;
}
}  // namespace

extern "C" int ceos_sur_set_params(void* handle, const float* theta) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !theta) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    CKS(cudaMemcpyAsync(s->theta, theta, sizeof(float) * kNParams, cudaMemcpyHostToDevice, s->stream));
    CKS(cudaMemsetAsync(s->m1, 0, sizeof(float) * kNParams, s->stream));
    CKS(cudaMemsetAsync(s->m2, 0, sizeof(float) * kNParams, s->stream));
    CKS(cudaMemsetAsync(s->grad, 0, sizeof(float) * kNParams, s->stream));
    CKS(cudaMemsetAsync(s->ctr, 0, sizeof(int) * 2, s->stream));
    s->step = 0;
    int rc = refresh(s);
    if (rc) return rc;
    CKS(cudaStreamSynchronize(s->stream));
    return 0;
}

extern "C" int ceos_sur_get_params(void* handle, float* theta) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !theta) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    CKS(cudaMemcpyAsync(theta, s->theta, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, s->stream));
    CKS(cudaStreamSynchronize(s->stream));
    return 0;
}

extern "C" int ceos_sur_set_scaling(void* handle, const double* scales, const double* lo, const double* hi) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !scales) return CEOS_E_ARG;
    for (int k = 0; k < 4; ++k) s->scales[k] = (float)scales[k];
    if (!(s->scales[0] > 0.f) || !(s->scales[1] > 0.f) || !(s->scales[3] > 0.f)) return CEOS_E_ARG;
    if (lo && hi)
        for (int k = 0; k < kIn; ++k) { s->lo[k] = (float)lo[k]; s->hi[k] = (float)hi[k]; }
    float b[2 * kIn];
    std::copy(s->lo, s->lo + kIn, b);
    std::copy(s->hi, s->hi + kIn, b + kIn);
    CKS(cudaSetDevice(s->device));
    CKS(cudaMemcpy(s->box, b, sizeof(b), cudaMemcpyHostToDevice));
    return 0;
}

// Gradient of the Sobolev loss over one batch (x [n][7] normalised inputs, t [n][6] targets of
// de/dx, w [6] component weights, sw [n] sample weights or NULL): grad [n_params] and the loss.
extern "C" int ceos_sur_gradient(void* handle, int n, const float* x, const float* t, const float* w, const float* sw,
                                 float* grad, double* loss) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || n < 1 || n > s->cap || !x || !t || !w || !grad) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    float* dX = nullptr;
    CKS(cudaMalloc(&dX, sizeof(float) * kIn * (size_t)n));
    cudaMemcpyAsync(dX, x, sizeof(float) * kIn * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(s->T, t, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(s->w6, w, sizeof(float) * 6, cudaMemcpyHostToDevice, s->stream);
    {
        std::vector<float> ones;
        if (!sw) ones.assign(n, 1.f);
        cudaMemcpy(s->Sw, sw ? sw : ones.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
    }
    cudaMemsetAsync(s->grad, 0, sizeof(float) * kNParams, s->stream);
    cudaMemsetAsync(s->loss, 0, sizeof(double), s->stream);
    int rc = grad_device(s, n, dX);
    if (!rc) {
        cudaMemcpyAsync(grad, s->grad, sizeof(float) * kNParams, cudaMemcpyDeviceToHost, s->stream);
        if (loss) cudaMemcpyAsync(loss, s->loss, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
        cudaMemsetAsync(s->grad, 0, sizeof(float) * kNParams, s->stream);
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    cudaFree(dX);
    if (rc) return rc;
    CKS(e);
    return gemm_error(s);
}

// Adam training on n samples (x [n][7], t [n][6], w [6], sample weights sw [n] or NULL): epochs
// passes over a per-epoch
// shuffle (seeded), mini-batches of `batch` (<= capacity; the last partial batch of an epoch is
// dropped), learning rate decaying geometrically from lr0 to lr1 over all steps.  One step
// (batch gather, the four passes, weight gradients, Adam) is captured once into a CUDA graph
// and replayed.  loss_hist[epochs] = mean batch loss of each epoch.
extern "C" int ceos_sur_train(void* handle, int n, const float* x, const float* t, const float* w, const float* sw,
                              int epochs, int batch, double lr0, double lr1, unsigned seed, double* loss_hist) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !x || !t || !w || epochs < 1 || batch < 1 || batch > s->cap || n < batch || !(lr0 > 0) || !(lr1 > 0))
        return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    const int nbatch = n / batch;
    const double decay = std::pow(lr1 / lr0, 1.0 / std::max(1, epochs * nbatch - 1));
    float *dXall = nullptr, *dTall = nullptr, *dX = nullptr, *dSw = nullptr;
    int* didx = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int rc = 0;
    auto fail = [&](const char* what) {
        if (s->msg.empty()) s->msg = what;
        if (!rc) rc = CEOS_E_CUDA;
    };
    if (cudaMalloc(&dXall, sizeof(float) * kIn * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dTall, sizeof(float) * 6 * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dX, sizeof(float) * kIn * (size_t)batch) != cudaSuccess ||
        cudaMalloc(&didx, sizeof(int) * (size_t)n) != cudaSuccess ||
        cudaMalloc(&dSw, sizeof(float) * (size_t)n) != cudaSuccess)
        fail("training buffers");
    if (!rc) {
        cudaMemcpyAsync(dXall, x, sizeof(float) * kIn * (size_t)n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(dTall, t, sizeof(float) * 6 * (size_t)n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(s->w6, w, sizeof(float) * 6, cudaMemcpyHostToDevice, st);
        {
            std::vector<float> ones;
            if (!sw) ones.assign(n, 1.f);
            cudaMemcpy(dSw, sw ? sw : ones.data(), sizeof(float) * (size_t)n, cudaMemcpyHostToDevice);
        }
        // capture one step
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            fail("begin capture");
        } else {
            step_kernel<<<1, 1, 0, st>>>(s->ctr, (float)lr0, (float)decay, 0.9f, 0.999f, s->hp);
            gather_rows_kernel<<<(batch + 255) / 256, 256, 0, st>>>(batch, s->ctr, didx, dXall, dTall, dSw, dX, s->T,
                                                                    s->Sw);
            const int r2 = grad_device(s, batch, dX);
            adam_kernel<<<(kNParams + 255) / 256, 256, 0, st>>>(s->theta, s->grad, s->m1, s->m2, s->hp, 0.9f, 0.999f,
                                                                1e-8f, s->Wb1, s->Wb, s->WbT);
            advance_kernel<<<1, 1, 0, st>>>(s->ctr, batch);
            const cudaError_t e = cudaStreamEndCapture(st, &graph);
            if (r2 || e != cudaSuccess || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess)
                fail("training step graph capture");
        }
    }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937 rng(seed);
    for (int ep = 0; ep < epochs && !rc; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        cudaMemcpyAsync(didx, perm.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(s->ctr + 1, 0, sizeof(int), st);
        cudaMemsetAsync(s->loss, 0, sizeof(double), st);
        for (int b = 0; b < nbatch && !rc; ++b)
            if (cudaGraphLaunch(exec, st) != cudaSuccess) fail("graph launch");
        double lsum = 0.0;
        cudaMemcpyAsync(&lsum, s->loss, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) fail("training step");  // perm reused next epoch
        if (loss_hist) loss_hist[ep] = lsum / nbatch;
    }
    s->step += epochs * nbatch;
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (!rc) {
        transpose_f32_kernel<<<(3 * kH * kH + 255) / 256, 256, 0, st>>>(s->theta, s->WT);
        if (cudaStreamSynchronize(st) != cudaSuccess) fail("transpose");
    }
    cudaFree(didx);
    cudaFree(dSw);
    cudaFree(dX);
    cudaFree(dTall);
    cudaFree(dXall);
    return rc ? rc : gemm_error(s);
}

// Select the 128-wide layer GEMMs of training: 1 tcgen05 tensor cores (the default), 0 mma.sync.
extern "C" int ceos_sur_set_gemm(void* handle, int path) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || path < 0 || path > 1) return CEOS_E_ARG;
    s->gemm_path = path;
    return 0;
}

namespace {
int launch_infer(Sur* s, InferArgs& a, cudaStream_t st) {
    a.theta = s->theta;
    a.WT = s->WT;
    a.sC = s->scales[0];
    a.sW = s->scales[1];
    a.vf0 = s->scales[2];
    a.svf = s->scales[3];
    a.lo = s->box;
    a.hi = s->box + kIn;
    if (s->s0_on) {
        a.s0tab = s->s0tab;
        a.n_tab = kTab;
        a.tab_lo = s->tab_lo;
        a.tab_hi = s->tab_hi;
    }
    CKS(cudaFuncSetAttribute(infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const int tiles = (a.n + kTP - 1) / kTP;
    infer_kernel<<<std::max(1, std::min(tiles, sms)), 256, kInferSmem, st>>>(a);
    CKS(cudaGetLastError());
    return 0;
}
}  // namespace

// Host-facing inference: C6 [n][6] (C11, C22, C33, C12, C23, C13), vf [n] -> S [n][6],
// material tangent [n][36] (Voigt tensor components), out_of_range [n] (any may be NULL).
extern "C" int ceos_sur_evaluate(void* handle, int n, const double* C6, const double* vf, double* S, double* Cm,
                                 int* out_of_range) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || n < 1 || !C6 || !vf) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    double *dC = nullptr, *dv = nullptr, *dS = nullptr, *dCm = nullptr;
    int* dfl = nullptr;
    CKS(cudaMalloc(&dC, sizeof(double) * 6 * (size_t)n));
    CKS(cudaMalloc(&dv, sizeof(double) * (size_t)n));
    CKS(cudaMalloc(&dS, sizeof(double) * 6 * (size_t)n));
    CKS(cudaMalloc(&dCm, sizeof(double) * 36 * (size_t)n));
    CKS(cudaMalloc(&dfl, sizeof(int) * (size_t)n));
    cudaMemcpyAsync(dC, C6, sizeof(double) * 6 * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(dv, vf, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, s->stream);
    InferArgs a{};
    a.n = n;
    a.C6 = dC;
    a.vf = dv;
    a.vf_mod = n;
    a.S = dS;
    a.Cm = dCm;
    a.flag = dfl;
    int rc = launch_infer(s, a, s->stream);
    if (!rc) {
        if (S) cudaMemcpyAsync(S, dS, sizeof(double) * 6 * (size_t)n, cudaMemcpyDeviceToHost, s->stream);
        if (Cm) cudaMemcpyAsync(Cm, dCm, sizeof(double) * 36 * (size_t)n, cudaMemcpyDeviceToHost, s->stream);
        if (out_of_range) cudaMemcpyAsync(out_of_range, dfl, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s->stream);
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    cudaFree(dC); cudaFree(dv); cudaFree(dS); cudaFree(dCm); cudaFree(dfl);
    if (rc) return rc;
    CKS(e);
    return 0;
}

// Make the undeformed state stress-free: tabulate the network's S at C = I for vf in [vf_lo, vf_hi]
// and subtract it (linearly interpolated in vf) from every later stress.  This subtracts a term
// linear in C from the energy, so the tangent is unchanged.  Call again after training.
extern "C" int ceos_sur_set_reference(void* handle, double vf_lo, double vf_hi) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !(vf_hi > vf_lo)) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    s->s0_on = 0;
    std::vector<double> C6(6 * kTab, 0.0), vf(kTab), S0(6 * kTab);
    for (int i = 0; i < kTab; ++i) {
        C6[6 * i] = C6[6 * i + 1] = C6[6 * i + 2] = 1.0;
        vf[i] = vf_lo + (vf_hi - vf_lo) * i / (kTab - 1);
    }
    int rc = ceos_sur_evaluate(handle, kTab, C6.data(), vf.data(), S0.data(), nullptr, nullptr);
    if (rc) return rc;
    if (!s->s0tab) CKS(cudaMalloc(&s->s0tab, sizeof(double) * 6 * kTab));
    CKS(cudaMemcpy(s->s0tab, S0.data(), sizeof(double) * 6 * kTab, cudaMemcpyHostToDevice));
    s->tab_lo = vf_lo;
    s->tab_hi = vf_hi;
    s->s0_on = 1;
    return 0;
}

// Device-side material evaluation for the element loop: F [9][ldF] (row-major per point,
// point q = gp * n_elem + e, FP64), vf [n_elem] -> Cauchy stress and spatial tangent written to
// the external-material state state[(v*8 + gp)*ld + e] (v < 6 stress, 6.. the 21 upper entries
// of D), FP32 or FP64; flags [8 n_elem] = 1 where the point is outside the training box.
extern "C" int ceos_sur_material_device(void* handle, int n_elem, const double* F, long long ldF, const double* vf,
                                        void* state, int state_f32, long long ld, int* flags, void* stream) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || n_elem < 1 || !F || ldF < 8LL * n_elem || !vf || !state || ld < n_elem) return CEOS_E_ARG;
    CKS(cudaSetDevice(s->device));
    InferArgs a{};
    a.n = 8 * n_elem;
    a.F = F;
    a.ldF = ldF;
    a.vf = vf;
    a.vf_mod = n_elem;
    a.flag = flags;
    a.state = state;
    a.state_f32 = state_f32;
    a.ld = ld;
    a.n_elem = n_elem;
    return launch_infer(s, a, static_cast<cudaStream_t>(stream));
}

extern "C" int ceos_sur_message(void* handle, char* msg, int len) {
    Sur* s = static_cast<Sur*>(handle);
    if (!s || !msg || len < 1) return CEOS_E_ARG;
    std::snprintf(msg, len, "%s", s->msg.c_str());
    return 0;
}

extern "C" void ceos_sur_destroy(void* handle) { delete static_cast<Sur*>(handle); }
