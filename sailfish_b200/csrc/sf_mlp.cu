// Learned vertical-mixing closure: a per-column MLP (5 dense layers of width 128, GELU between
// them) with BF16 operands and FP32 accumulation on the Blackwell tensor cores (tcgen05.mma
// with the accumulator in tensor memory), its training (forward with saved activations,
// backward, Adam) and the feature / output mapping to the model state.
//
// The reference has no counterpart: its vertical mixing is a fixed analytic profile and its
// GLS closure exists only as untranslated ROMS Fortran.  The network stands in for the GLS
// corrector (sf_gls.cuh); plain GLS stays the fallback for columns outside the training range
// and the reference that the network's error is measured against.
//
// All dense products go through one tile routine, D[128x128] (TMEM, FP32) = A[128xK] B[128xK]^T
// with A and B staged in shared memory as BF16 in the K-major, no-swizzle "core matrix" layout
// (8 rows x 16 bytes per core matrix), so forward layers (A = activations, B = W), input
// gradients (A = G, B = W^T) and weight gradients (A = G^T, B = X^T) only differ in how the
// operands are read from global memory while they are staged.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <type_traits>

#include "sf_internal.h"

namespace sf {
namespace mlp {

constexpr int kTile = 128;         // rows of an output tile (MMA M) and width of every layer
constexpr int kThreads = 128;      // 4 warps: warp w owns TMEM lanes 32w..32w+31
constexpr uint32_t kTmemCols = 128;
constexpr size_t kGemmSmem = 2 * 128 * 128 * 2;   // A and B tiles, BF16

// ---- PTX wrappers ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major, no swizzle (tcgen05 "version 1" format): start
// address, leading byte offset (between the two 8-element K halves of a K=16 step), stride
// byte offset (between 8-row groups), all in 16-byte units.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100
    return d;                 // base offset 0, legacy LBO mode, layout SWIZZLE_NONE (0)
}

// Instruction descriptor, kind::f16: D FP32, A and B BF16, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols));
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kIdesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(mbar)));
}
__device__ __forceinline__ void mbar_init(uint64_t *mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
}
// Bounded wait on an mbarrier phase; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
    const uint32_t a = smem_u32(mbar);
    for (int it = 0; it < (1 << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity));
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}
// Row lane, 32 consecutive FP32 columns from registers (32x32b.x32), and the wait for them.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const float *v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
        "%30, %31, %32};" ::"r"(taddr),
        "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]),
        "f"(v[8]), "f"(v[9]), "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15]),
        "f"(v[16]), "f"(v[17]), "f"(v[18]), "f"(v[19]), "f"(v[20]), "f"(v[21]), "f"(v[22]), "f"(v[23]),
        "f"(v[24]), "f"(v[25]), "f"(v[26]), "f"(v[27]), "f"(v[28]), "f"(v[29]), "f"(v[30]), "f"(v[31])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// The accumulator columns n0..n0+31 of this thread's row set to the bias: the products then add
// onto it (the layer's pre-activation is bias + sum, accumulated by the tensor cores).
__device__ __forceinline__ void tmem_bias32(uint32_t taddr, const float *bias32) {
    float v[32];
#pragma unroll
    for (int k = 0; k < 32; k += 4) {
        const float4 q = *reinterpret_cast<const float4 *>(bias32 + k);
        v[k] = q.x;
        v[k + 1] = q.y;
        v[k + 2] = q.z;
        v[k + 3] = q.w;
    }
    tmem_st32(taddr, v);
}

// Element (r, k) of a 128 x 128 BF16 tile in the core-matrix layout: 16 core matrices of
// 8 x 8 along K per 8-row group; a core matrix is 8 rows of 16 contiguous bytes.
__device__ __forceinline__ int cm_index(int r, int k) {
    return (((r >> 3) * 16 + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}
constexpr uint32_t kLBO = 128;       // next 8-element K half: next core matrix
constexpr uint32_t kSBO = 16 * 128;  // next 8-row group

// A matrix in global memory read as element (row, k) = p[row*rs + k*ks], FP32 or BF16.
struct Mat {
    const void *p;
    int bf16;
    long rs, ks;
    long rows, cols;   // valid extent; outside it the staged value is 0
    __device__ __forceinline__ float at(long r, long k) const {
        if (r >= rows || k >= cols) return 0.f;
        const long o = r * rs + k * ks;
        return bf16 ? __bfloat162float(((const __nv_bfloat16 *)p)[o]) : ((const float *)p)[o];
    }
};

// The closure's feature and output maps use the hardware approximations (relative error
// ~2^-21, far below the BF16 rounding of the network's operands); features for training and
// for inference go through the same functions.
__device__ __forceinline__ float flog10(float x) { return __log10f(x); }
__device__ __forceinline__ float fexp10(float x) { return __exp10f(x); }

__device__ __forceinline__ float gelu(float x) {   // tanh form of the GELU
    const float c = 0.7978845608028654f;           // sqrt(2/pi)
    return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float c = 0.7978845608028654f;
    const float u = c * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * x * x);
}
// Activation codes of k_gemm and the backward pass: 0 none, 1 GELU, 2 ReLU.
constexpr int kActNone = 0, kActGelu = 1, kActRelu = 2;
__device__ __forceinline__ float act_apply(float z, int act) {
    return act == kActGelu ? gelu(z) : (act == kActRelu ? fmaxf(z, 0.f) : z);
}
inline int act_code(const sf_mlp_params *w) { return w->act == SF_MLP_RELU ? kActRelu : kActGelu; }

// D tile (blockIdx.x) = A[m0:m0+128, 0:K] B[0:128, 0:K]^T, K a multiple of 16, staged 128 K
// at a time.  Epilogue: v = D + bias; Z[r, n] = v (optional); O[r, n] = act(v).
__global__ void __launch_bounds__(kThreads) k_gemm(Mat A, Mat B, long Mrows, int K,
                                                   const float *__restrict__ bias, int act,
                                                   float *__restrict__ O, long ldo,
                                                   float *__restrict__ Z, long ldz, int *err) {
    extern __shared__ __align__(1024) unsigned char dsm[];
    __nv_bfloat16 *sA = reinterpret_cast<__nv_bfloat16 *>(dsm);
    __nv_bfloat16 *sB = sA + kTile * kTile;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long m0 = (long)blockIdx.x * kTile;
    if (warp == 0) tmem_alloc(&tmem_base);
    if (tid == 0) {
        mbar_init(&mbar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K; k0 += kTile) {
        const int kc = min(kTile, K - k0);
        for (int e = tid; e < kTile * kc; e += kThreads) {
            const int r = e / kc, k = e - r * kc;
            sA[cm_index(r, k)] = __float2bfloat16_rn(A.at(m0 + r, k0 + k));
            sB[cm_index(r, k)] = __float2bfloat16_rn(B.at(r, k0 + k));
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int s = 0; s < kc / 16; ++s)
                mma_bf16(tmem, sdesc(a0 + s * 256, kLBO, kSBO), sdesc(b0 + s * 256, kLBO, kSBO),
                         (k0 > 0 || s > 0) ? 1u : 0u);
            mma_commit(&mbar);
        }
        if (!mbar_wait(&mbar, phase)) ok = false;
        phase ^= 1;
        fence_after();
        __syncthreads();
        if (!ok) break;
    }
    if (ok) {
        const long r = m0 + warp * 32 + lane;
        for (int c = 0; c < kTile / 32; ++c) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c * 32, v);
            if (r < Mrows) {
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const int n = c * 32 + k;
                    const float z = v[k] + (bias ? bias[n] : 0.f);
                    if (Z) Z[r * ldz + n] = z;
                    O[r * ldo + n] = act_apply(z, act);
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem);
}

// G = dA * act'(Z) (elementwise, n x 128; ReLU' taken as 0 at 0)
__global__ void k_act_back(long n, const float *__restrict__ dA, const float *__restrict__ Z,
                           float *__restrict__ G, int act) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n * kTile) {
        const float z = Z[e];
        G[e] = dA[e] * (act == kActRelu ? (z > 0.f ? 1.f : 0.f) : gelu_grad(z));
    }
}

// db[j] = sum_m G[m, j]
__global__ void k_colsum(long n, const float *__restrict__ G, float *__restrict__ db) {
    const int j = threadIdx.x;
    float s = 0.f;
    for (long m = blockIdx.x; m < n; m += gridDim.x) s += G[m * kTile + j];
    atomicAdd(&db[j], s);
}

// MSE on the first nvalid outputs: dY = 2 (Y - T) / (n * nvalid), loss accumulated into *loss.
__global__ void k_mse(long n, int nvalid, const float *__restrict__ Y, const float *__restrict__ T,
                      float *__restrict__ dY, float *loss) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (e < n * kTile) {
        const int j = (int)(e % kTile);
        float g = 0.f;
        if (j < nvalid) {
            const float d = Y[e] - T[e];
            g = 2.f * d / (float)(n * nvalid);
            l = d * d / (float)(n * nvalid);
        }
        dY[e] = g;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
}

// Adam step on FP32 master weights; refreshes the BF16 copy used by the tensor cores.
__global__ void k_adam(long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, __nv_bfloat16 *__restrict__ wb, float lr, float b1,
                       float b2, float c1, float c2, float eps) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const float gg = g[e];
    const float mm = b1 * m[e] + (1.f - b1) * gg;
    const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
    m[e] = mm;
    v[e] = vv;
    const float ww = w[e] - lr * (mm / c1) / (sqrtf(vv / c2) + eps);
    w[e] = ww;
    if (wb) wb[e] = __float2bfloat16_rn(ww);
}

// ---- fused inference -----------------------------------------------------------------------
// All SF_MLP_LAYERS layers of a 128-row tile in one pass: the BF16 weights of every layer stay
// in shared memory for the life of the (persistent, one per SM) CTA, the activations of the
// tile stay in shared memory between layers, and only the input rows are read and the output
// rows written.  Per layer: 8 MMAs (K = 128) into the TMEM accumulator, then 8 warps read it
// back (warp w: TMEM lanes 32(w%4).., columns 64(w/4)..), add the bias, apply the GELU and
// write the next layer's BF16 operand in place of the current one.
constexpr int kInferThreads = 256;
constexpr size_t kInferSmem = (size_t)(1 + SF_MLP_LAYERS) * kTile * kTile * 2;

struct InferW {
    const __nv_bfloat16 *W[SF_MLP_LAYERS];
    const float *b[SF_MLP_LAYERS];
};

// GELU, tanh form, with the hardware tanh approximation (relative error ~2^-11, below the BF16
// rounding of the activations it feeds).
__device__ __forceinline__ float gelu_fast(float x) {
    const float c = 0.7978845608028654f;
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(c * (x + 0.044715f * x * x * x)));
    return 0.5f * x * (1.f + t);
}

template <int ACT>
__device__ __forceinline__ float act_fast(float x) {
    if constexpr (ACT == kActRelu) return fmaxf(x, 0.f);
    else return gelu_fast(x);
}

// BF16 pair {act(lo), act(hi)} (lo in the low half); for ReLU one conversion with clamping.
template <int ACT>
__device__ __forceinline__ uint32_t pack_act2(float lo, float hi) {
    if constexpr (ACT == kActRelu) {
        uint32_t d;
        asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
        return d;
    } else {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(act_fast<ACT>(lo), act_fast<ACT>(hi));
        return *reinterpret_cast<const uint32_t *>(&b2);
    }
}

// act(v) of 32 consecutive pre-activations of row r (the bias is already in them), as the next
// layer's BF16 operand: four 16-byte stores, one per core-matrix row segment.
template <int ACT>
__device__ __forceinline__ void store_act8x4(__nv_bfloat16 *sA, int r, int n0, const float *v) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t pk[4];
#pragma unroll
        for (int h = 0; h < 4; ++h) pk[h] = pack_act2<ACT>(v[8 * q + 2 * h], v[8 * q + 2 * h + 1]);
        *reinterpret_cast<uint4 *>(&sA[cm_index(r, n0 + 8 * q)]) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
}

template <int ACT>
__global__ void __launch_bounds__(kInferThreads, 1) k_infer(InferW w, long n,
                                                            const float *__restrict__ X,
                                                            float *__restrict__ Y, int *err) {
    extern __shared__ __align__(1024) unsigned char dsm[];
    __nv_bfloat16 *sA = reinterpret_cast<__nv_bfloat16 *>(dsm);
    __nv_bfloat16 *sW = sA + kTile * kTile;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ __align__(16) float sbias[SF_MLP_LAYERS][kTile];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tmem_alloc(&tmem_base);
    if (tid == 0) {
        mbar_init(&mbar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    for (int l = 0; l < SF_MLP_LAYERS; ++l) {
        for (int e = tid; e < kTile * kTile; e += kInferThreads)
            sW[l * kTile * kTile + cm_index(e >> 7, e & 127)] = w.W[l][e];
        for (int e = tid; e < kTile; e += kInferThreads) sbias[l][e] = w.b[l] ? w.b[l][e] : 0.f;
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = tmem_base;
    const int rl = (warp & 3) * 32 + lane;        // tile row of this thread in the epilogue
    const int cb = (warp >> 2) * 64;              // first of its 64 columns
    const uint32_t trow = (uint32_t)((warp & 3) * 32) << 16;
    uint32_t phase = 0;
    bool ok = true;
    const long ntiles = (n + kTile - 1) / kTile;
    for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const long m0 = t * kTile;
        // stage the input tile: 16 float4 in flight per thread, then BF16 into the operand
        {
            float4 q[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int e4 = tid + u * kInferThreads;   // float4 index in the 128 x 32 tile
                const long r = m0 + (e4 >> 5);
                q[u] = r < n ? reinterpret_cast<const float4 *>(X + r * kTile)[e4 & 31]
                             : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int e4 = tid + u * kInferThreads;
                const int r = e4 >> 5, k = (e4 & 31) * 4;
                sA[cm_index(r, k + 0)] = __float2bfloat16_rn(q[u].x);
                sA[cm_index(r, k + 1)] = __float2bfloat16_rn(q[u].y);
                sA[cm_index(r, k + 2)] = __float2bfloat16_rn(q[u].z);
                sA[cm_index(r, k + 3)] = __float2bfloat16_rn(q[u].w);
            }
        }
        for (int l = 0; l < SF_MLP_LAYERS; ++l) {
            // the layer's bias into the accumulator (this thread's row and 64 columns)
            for (int c = 0; c < 2; ++c) tmem_bias32(tmem + trow + cb + c * 32, sbias[l] + cb + c * 32);
            tmem_wait_st();
            fence_before();
            fence_proxy_async();
            __syncthreads();
            if (tid == 0) {
                fence_after();
                const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sW + l * kTile * kTile);
                for (int s = 0; s < kTile / 16; ++s)
                    mma_bf16(tmem, sdesc(a0 + s * 256, kLBO, kSBO), sdesc(b0 + s * 256, kLBO, kSBO), 1u);
                mma_commit(&mbar);
            }
            const bool done = mbar_wait(&mbar, phase);
            phase ^= 1;
            fence_after();
            if (__syncthreads_or(!done)) {
                ok = false;
                break;
            }
            const bool last = l == SF_MLP_LAYERS - 1;
            const long r = m0 + rl;
            for (int c = 0; c < 2; ++c) {
                float v[32];
                tmem_ld32(tmem + trow + cb + c * 32, v);
                const int n0 = cb + c * 32;
                if (!last) {
                    store_act8x4<ACT>(sA, rl, n0, v);
                } else if (r < n) {
                    float4 *y = reinterpret_cast<float4 *>(Y + r * kTile + n0);
#pragma unroll
                    for (int k = 0; k < 8; ++k) y[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
                }
            }
            fence_before();
        }
    }
    if (!ok && tid == 0) atomicExch(err, 1);
    fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem);
}

}  // namespace mlp
}  // namespace sf

// =============================================================================================
// Feature extraction and output mapping (model state <-> MLP rows), one row per water column
// =============================================================================================
namespace sf {
namespace mlp {

// Rho-interior water column (the interior rho points of mod_cppkernels.cpp:20).
__device__ __forceinline__ bool column_(int i, int j, int I, int J) {
    return !(i == 0 || i == I - 1 || j == 0 || j == J - 1);
}

// mask[p] = 1 for a rho-interior column whose feature row leaves the box [lo, hi] in any of
// its first nfeat features (a column outside the range the network was trained on), else 0.
__global__ void k_range_mask(long s2, int I, int J, int nfeat, const float *__restrict__ X,
                             const float *__restrict__ lo, const float *__restrict__ hi,
                             uint8_t *__restrict__ mask) {
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s2) return;
    uint8_t out = 0;
    if (column_((int)(p % I), (int)(p / I), I, J)) {
        const float *x = X + p * kTile;
        for (int k = 0; k < nfeat; ++k)
            if (!(x[k] >= lo[k] && x[k] <= hi[k])) out = 1;   // NaN counts as outside
    }
    mask[p] = out;
}

// Feature row of the column at p (rho-interior), nl = N-1 interior W levels: log-scaled shear^2
// at levels 1..N-1 in x[0, nl), sign-preserving log-scaled N^2 in x[nl, 2nl), then log10 of
// the surface friction velocity squared, the surface buoyancy flux (0: no heat flux in these
// basins) and log10 of the depth in x[2nl], x[2nl+1], x[2nl+2]; the rest of the 128 are 0.
template <typename R>
__global__ void k_features(Geo<R> g, const R *__restrict__ u, const R *__restrict__ v,
                           const R *__restrict__ z_r, const R *__restrict__ bvf,
                           const R *__restrict__ sustr, const R *__restrict__ svstr,
                           float *__restrict__ X) {
    const int pi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (pi >= g.s2) return;
    const long p = pi, I = g.I, s2 = g.s2;
    const int N = g.N;
    float *x = X + p * kTile;
    for (int k = 0; k < kTile; ++k) x[k] = 0.f;
    const int i = pi % g.I, j = pi / g.I;
    if (!column_(i, j, g.I, g.J)) return;
#define AT(A, k, q) ((float)(A)[(long)(k) * s2 + (q)])
    const int nl = N - 1;   // interior W levels; 2 nl + 3 <= 128 is checked by the caller
    for (int k = 1; k < N; ++k) {
        const float cff = __fdividef(0.5f, AT(z_r, k, p) - AT(z_r, k - 1, p));
        const float du = (AT(u, k, p) - AT(u, k - 1, p)) + (AT(u, k, p + 1) - AT(u, k - 1, p + 1));
        const float dv = (AT(v, k, p) - AT(v, k - 1, p)) + (AT(v, k, p + I) - AT(v, k - 1, p + I));
        const float sh2 = (cff * du) * (cff * du) + (cff * dv) * (cff * dv);
        const float n2 = AT(bvf, k, p);
        x[k - 1] = flog10(sh2 + 1e-12f);
        x[nl + k - 1] = copysignf(flog10(1.f + fabsf(n2) * 1e8f), n2);
    }
    const float su = (float)(sustr[p] + sustr[p + 1]), sv = (float)(svstr[p] + svstr[p + I]);
    x[2 * nl] = flog10(0.5f * sqrtf(su * su + sv * sv) + 1e-10f);
    x[2 * nl + 1] = 0.f;
    x[2 * nl + 2] = flog10((float)g.hd[p]);
#undef AT
}

// Akv, Akt at interior W levels 1..N-1 from the outputs y[0, nl) and y[nl, 2nl) (log10,
// clipped to [-6, -1]); columns flagged in `fallback` (non-zero) keep the values in Akv/Akt.
template <typename R>
__global__ void k_apply(Geo<R> g, const float *__restrict__ Y, const uint8_t *__restrict__ fallback,
                        R *__restrict__ Akv, R *__restrict__ Akt) {
    const int pi = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (pi >= g.s2) return;
    const int i = pi % g.I, j = pi / g.I;
    if (!column_(i, j, g.I, g.J)) return;
    if (fallback && fallback[pi]) return;
    const long p = pi, s2 = g.s2;
    const float *y = Y + p * kTile;
    const int nl = g.N - 1;
    for (int k = 1; k < g.N; ++k) {
        Akv[(long)k * s2 + p] = (R)fexp10(fminf(fmaxf(y[k - 1], -6.f), -1.f));
        Akt[(long)k * s2 + p] = (R)fexp10(fminf(fmaxf(y[nl + k - 1], -6.f), -1.f));
    }
}


// ---- the closure: feature rows, then the network over row tiles ------------------------------
// k_closure_rows: one thread per flat column (full occupancy, so the level loads of many columns
// are in flight): it marches up the column carrying the level below in registers (6 loads per
// level), writes the BF16 feature row straight into a 128-row tile stored in the MMA operand's
// core-matrix layout (16-byte stores), checks the row against [lo, hi] and flags/lists the
// columns outside it.  k_closure_mlp: persistent, one CTA per SM holding every layer's weights
// in shared memory; each tile's operand arrives with one bulk copy (cp.async.bulk, 32 KB),
// issued for the next tile as soon as the last layer's products have read the current one, so
// it overlaps the output epilogue; the epilogue writes Akv/Akt level by level (lanes along the
// columns: coalesced) for the interior columns in range.
template <typename R>
__global__ void __launch_bounds__(128) k_closure_rows(Geo<R> g, const R *__restrict__ u,
        const R *__restrict__ v, const R *__restrict__ z_r, const R *__restrict__ bvf,
        const R *__restrict__ sustr, const R *__restrict__ svstr, int nfeat,
        const float *__restrict__ lo, const float *__restrict__ hi, uint8_t *__restrict__ fallback,
        int *__restrict__ flist, int *__restrict__ fcount, __nv_bfloat16 *__restrict__ Xt, long nrows) {
    __shared__ float slo[kTile], shi[kTile];   // the range box, read by every feature check
    for (int f = threadIdx.x; f < kTile; f += blockDim.x) {
        slo[f] = f < nfeat ? lo[f] : 0.f;
        shi[f] = f < nfeat ? hi[f] : 0.f;
    }
    __syncthreads();
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nrows) return;
    const long s2 = g.s2, I = g.I;
    const int nl = g.N - 1;
    __nv_bfloat16 *tile = Xt + (p / kTile) * (long)(kTile * kTile);
    const int r = (int)(p % kTile);
    const bool col = p < s2 && column_((int)(p % g.I), (int)(p / g.I), g.I, g.J);
    bool out = false;
    // column pointers, advanced one level (s2) per shear feature; the level below in registers
    const R *zc = z_r + p, *uc = u + p, *vc = v + p;
    float zb = 0.f, ub = 0.f, ube = 0.f, vb = 0.f, vbn = 0.f;
    if (col) {
        zb = (float)zc[0];
        ub = (float)uc[0];
        ube = (float)uc[1];
        vb = (float)vc[0];
        vbn = (float)vc[I];
    }
    auto shear = [&]() {   // feature of the next W level, carrying that level into registers
        zc += s2;
        uc += s2;
        vc += s2;
        const float zt = (float)zc[0], ut = (float)uc[0], ute = (float)uc[1];
        const float vt = (float)vc[0], vtn = (float)vc[I];
        const float cff = __fdividef(0.5f, zt - zb);
        const float du = (ut - ub) + (ute - ube), dv = (vt - vb) + (vtn - vbn);
        const float sh2 = (cff * du) * (cff * du) + (cff * dv) * (cff * dv);
        zb = zt;
        ub = ut;
        ube = ute;
        vb = vt;
        vbn = vtn;
        return flog10(sh2 + 1e-12f);
    };
    auto n2f = [&](int k) {
        const float n2 = (float)bvf[(long)k * s2 + p];
        return copysignf(flog10(1.f + fabsf(n2) * 1e8f), n2);
    };
    auto put8 = [&](int f0, const float *x) {
        uint32_t pk[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const __nv_bfloat162 b2 = __floats2bfloat162_rn(x[2 * q], x[2 * q + 1]);
            pk[q] = *reinterpret_cast<const uint32_t *>(&b2);
        }
        *reinterpret_cast<uint4 *>(tile + cm_index(r, f0)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    };
    auto check8 = [&](int f0, const float *x) {
#pragma unroll
        for (int h = 0; h < 8; ++h) {
            const int f = f0 + h;
            if (f < nfeat && !(x[h] >= slo[f] && x[h] <= shi[f])) out = true;
        }
    };
    int f0 = 0;
    if (col) {   // whole groups of 8 shear features (straight-line: the loads can be hoisted)
        for (; f0 + 8 <= nl; f0 += 8) {
            float x[8];
#pragma unroll
            for (int h = 0; h < 8; ++h) x[h] = shear();
            check8(f0, x);
            put8(f0, x);
        }
    }
    for (; f0 < kTile; f0 += 8) {
        float x[8];
        if (col && f0 >= nl && f0 + 8 <= 2 * nl) {   // whole groups of 8 N^2 features
#pragma unroll
            for (int h = 0; h < 8; ++h) x[h] = n2f(f0 + h - nl + 1);
        } else {
#pragma unroll
            for (int h = 0; h < 8; ++h) {
                const int f = f0 + h;
                float val = 0.f;
                if (col) {
                    if (f < nl) {
                        val = shear();
                    } else if (f < 2 * nl) {
                        val = n2f(f - nl + 1);
                    } else if (f == 2 * nl) {
                        const float su = (float)(sustr[p] + sustr[p + 1]);
                        const float sv = (float)(svstr[p] + svstr[p + I]);
                        val = flog10(0.5f * sqrtf(su * su + sv * sv) + 1e-10f);
                    } else if (f == 2 * nl + 2) {
                        val = flog10((float)g.hd[p]);
                    }
                }
                x[h] = val;
            }
        }
        if (col) check8(f0, x);
        put8(f0, x);
    }
    if (p < s2) {
        fallback[p] = out ? 1 : 0;
        if (out && flist) flist[atomicAdd(fcount, 1)] = (int)p;
    }
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)),
                 "r"(bytes));
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(mbar))
        : "memory");
}

// Two groups of 8 warps run their own tiles independently: group b takes this CTA's tiles
// 2i + b, with its own operand buffer, TMEM accumulator (columns 128b..) and mbarriers, and
// synchronises only its own 256 threads (named barrier 1 + b), so one group's epilogue runs
// while the other group's products are on the tensor cores.  Warp w of a group reads TMEM
// lanes 32(w%4).. (its rows) and columns 64((w/4)%2).. (64 outputs of a row per layer).
constexpr int kClosureThreads = 512;
constexpr size_t kClosureSmem = (size_t)(2 + SF_MLP_LAYERS) * kTile * kTile * 2;
constexpr uint32_t kTmemCols2 = 256;

__device__ __forceinline__ void tmem_alloc256(uint32_t *dst_smem) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(kTmemCols2));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc256(uint32_t taddr) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols2));
}
// Barrier over the 256 threads of named barrier `id`, returning whether any of them passed true.
__device__ __forceinline__ bool group_any(int id, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
        "barrier.red.or.pred q, %2, 256, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id)
        : "memory");
    return r != 0;
}

template <typename R, int ACT>
__global__ void __launch_bounds__(kClosureThreads, 1) k_closure_mlp(Geo<R> g, InferW w,
        const __nv_bfloat16 *__restrict__ Xt, long ntiles, const uint8_t *__restrict__ fallback,
        R *__restrict__ Akv, R *__restrict__ Akt, int *err) {
    extern __shared__ __align__(1024) unsigned char dsm[];
    __nv_bfloat16 *const sA0 = reinterpret_cast<__nv_bfloat16 *>(dsm);
    __nv_bfloat16 *const sW = sA0 + 2 * kTile * kTile;
    __shared__ __align__(8) uint64_t mbar[2], xbar[2];
    __shared__ uint32_t tmem_base;
    __shared__ __align__(16) float sbias[SF_MLP_LAYERS][kTile];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nl = g.N - 1;
    const long s2 = g.s2, G = gridDim.x;
    auto tile_of = [&](long q) { return (long)blockIdx.x + G * q; };   // this CTA's q-th tile
    if (warp == 0) tmem_alloc256(&tmem_base);
    if (tid == 0) {
        for (int b = 0; b < 2; ++b) {
            mbar_init(&mbar[b]);
            mbar_init(&xbar[b]);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
        fence_proxy_async();
        for (int b = 0; b < 2; ++b)   // each group's first operand, while the weights load
            if (tile_of(b) < ntiles)
                bulk_load(sA0 + b * kTile * kTile, Xt + tile_of(b) * kTile * kTile, kTile * kTile * 2,
                          &xbar[b]);
    }
    for (int l = 0; l < SF_MLP_LAYERS; ++l) {
        for (int e = tid; e < kTile * kTile; e += kClosureThreads)
            sW[l * kTile * kTile + cm_index(e >> 7, e & 127)] = w.W[l][e];
        for (int e = tid; e < kTile; e += kClosureThreads) sbias[l][e] = w.b[l] ? w.b[l][e] : 0.f;
    }
    fence_before();
    __syncthreads();
    fence_after();
    const int grp = warp >> 3, bar_id = 1 + grp;
    const bool issuer = (warp & 7) == 0 && lane == 0;
    __nv_bfloat16 *const sA = sA0 + grp * kTile * kTile;
    const uint32_t acc = tmem_base + (uint32_t)(grp * kTile);
    const int rl = (warp & 3) * 32 + lane;
    const int n0 = ((warp >> 2) & 1) * 64;
    const uint32_t tacc = acc + ((uint32_t)((warp & 3) * 32) << 16) + n0;
    uint32_t ph = 0, xph = 0;
    bool bad = false;    // this thread gave up a wait
    bool stop = false;   // the group gave up (uniform over the group: set from a vote)
    // the first layer's bias into this thread's accumulator columns; each epilogue then loads
    // the next layer's (or, after the last layer, the next tile's first layer's) bias into the
    // columns it has just read, and the products add onto it
    for (int c = 0; c < 2; ++c) tmem_bias32(tacc + c * 32, sbias[0] + n0 + c * 32);
    tmem_wait_st();
    fence_before();
    auto issue_mma = [&](int l) {   // the group's elected thread: layer l into its accumulator
        const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sW + l * kTile * kTile);
        for (int q = 0; q < kTile / 16; ++q)
            mma_bf16(acc, sdesc(a0 + q * 256, kLBO, kSBO), sdesc(b0 + q * 256, kLBO, kSBO), 1u);
        mma_commit(&mbar[grp]);
    };
    for (long i = 0;; ++i) {
        const long t = tile_of(2 * i + grp);
        if (t >= ntiles) break;
        bad = !mbar_wait(&xbar[grp], xph) || bad;   // this tile's operand landed
        xph ^= 1;
        // every thread's TMEM reads of the previous tile are done before this tile's products
        if (group_any(bar_id, bad)) {
            stop = true;
            break;
        }
        fence_after();
        if (issuer) issue_mma(0);
        const int p = (int)(t * kTile) + rl;   // the flat column of this thread's row
        bool apply = false;
        if (p < s2) {
            const int j = fdiv(p, g.dI);
            apply = column_(p - j * g.I, j, g.I, g.J) && !fallback[p];
        }
        for (int l = 0; l < SF_MLP_LAYERS; ++l) {
            const bool last = l == SF_MLP_LAYERS - 1;
            bad = !mbar_wait(&mbar[grp], ph) || bad;
            ph ^= 1;
            fence_after();
            if (last && issuer && !bad) {   // the products have read the operand: refill it
                const long nt = tile_of(2 * (i + 1) + grp);
                if (nt < ntiles) bulk_load(sA, Xt + nt * kTile * kTile, kTile * kTile * 2, &xbar[grp]);
            }
            if (!last) {
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float vv[32];
                    tmem_ld32(tacc + c * 32, vv);
                    store_act8x4<ACT>(sA, rl, n0 + c * 32, vv);
                    tmem_bias32(tacc + c * 32, sbias[l + 1] + n0 + c * 32);
                }
                tmem_wait_st();
                fence_before();
                fence_proxy_async();
                if (group_any(bar_id, bad)) {
                    stop = true;
                    break;
                }
                fence_after();
                if (issuer) issue_mma(l + 1);   // overlaps the other group's epilogue
            } else {
                // outputs n of this column: Akv at level n+1 for n < nl, then Akt at level
                // n-nl+1 for n < 2nl; the destination advances one level (s2) a step.  The TMEM
                // reads are warp-wide (every lane), the stores only for the columns updated.
                R *dst = n0 < nl ? Akv + (long)(n0 + 1) * s2 + p : Akt + (long)(n0 - nl + 1) * s2 + p;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    float vv[32];
                    tmem_ld32(tacc + c * 32, vv);
                    tmem_bias32(tacc + c * 32, sbias[0] + n0 + c * 32);
                    if (apply) {
#pragma unroll
                        for (int k = 0; k < 32; ++k) {
                            const int n = n0 + c * 32 + k;
                            if (n == nl) dst = Akt + s2 + p;
                            if (n < 2 * nl) __stcs(dst, (R)fexp10(fminf(fmaxf(vv[k], -6.f), -1.f)));
                            dst += s2;
                        }
                    }
                }
                tmem_wait_st();
                fence_before();
            }
        }
        if (stop) break;   // a last-layer wait that gave up is voted on at the next tile
    }
    if (bad) atomicExch(err, 1);
    if (stop && issuer) (void)mbar_wait(&xbar[grp], xph);   // a refill in flight (bounded)
    fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc256(tmem_base);
}

}  // namespace mlp
}  // namespace sf

// =============================================================================================
// C ABI
// =============================================================================================
namespace {
thread_local std::string g_mlp_err;
int mfail(int code, const char *msg) {
    g_mlp_err = msg;
    return code;
}
int mcuda(cudaError_t e, const char *where) {
    g_mlp_err = std::string(where) + ": " + cudaGetErrorString(e);
    return SF_ECUDA;
}
inline cudaStream_t S(sf_stream s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned nblk(long n, int b) { return (unsigned)((n + b - 1) / b); }
}  // namespace

using sf::mlp::Mat;
using sf::mlp::kTile;

extern "C" {

const char *sf_mlp_last_error(void) { return g_mlp_err.c_str(); }

int sf_mlp_gemm(int n_rows, int K, const void *A, int a_bf16, long a_rs, long a_ks,
                const void *B, int b_bf16, long b_rs, long b_ks, const float *bias, int act,
                float *O, long ldo, float *Z, long ldz, int *err, sf_stream s) {
    if (n_rows <= 0 || K <= 0 || K % 16 != 0) return mfail(SF_EINVAL, "K must be a positive multiple of 16");
    if (!A || !B || !O || !err) return mfail(SF_EINVAL, "null pointer");
    Mat a{A, a_bf16, a_rs, a_ks, n_rows, K}, b{B, b_bf16, b_rs, b_ks, kTile, K};
    // The raised shared-memory limit is a per-device function attribute: set it once on each
    // device the GEMM runs on.
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 != cudaSuccess) return mcuda(e0, "sf_mlp_gemm");
    if (dev < 0 || dev >= 64) return mfail(SF_EINVAL, "device ordinal out of range");
    if (!attr_set[dev]) {
        e0 = cudaFuncSetAttribute(sf::mlp::k_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)sf::mlp::kGemmSmem);
        if (e0 != cudaSuccess) return mcuda(e0, "sf_mlp_gemm");
        attr_set[dev] = true;
    }
    sf::mlp::k_gemm<<<nblk(n_rows, kTile), sf::mlp::kThreads, sf::mlp::kGemmSmem, S(s)>>>(
        a, b, n_rows, K, bias, act, O, ldo, Z, ldz, err);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_mlp_gemm");
}

int sf_mlp_forward(const sf_mlp_params *w, int n, const float *X, float *Y, float *acts,
                   float *pre, int *err, sf_stream s) {
    if (!w || !X || !Y || n <= 0) return mfail(SF_EINVAL, "bad argument");
    const long ld = kTile;
    const float *in = X;
    for (int l = 0; l < SF_MLP_LAYERS; ++l) {
        const bool last = l == SF_MLP_LAYERS - 1;
        float *out = last ? Y : (acts ? acts + (long)l * n * ld : nullptr);
        if (!out) return mfail(SF_EINVAL, "activation buffer required");
        float *z = pre ? pre + (long)l * n * ld : nullptr;
        const int rc = sf_mlp_gemm(n, kTile, in, 0, ld, 1, w->W[l], 1, ld, 1, w->b[l],
                                   last ? sf::mlp::kActNone : sf::mlp::act_code(w),
                                   out, ld, z, ld, err, s);
        if (rc) return rc;
        in = out;
    }
    return SF_OK;
}

int sf_mlp_backward(const sf_mlp_params *w, int n, const float *X, const float *acts,
                    const float *pre, const float *dY, float *const *dW, float *const *db,
                    float *work, int *err, sf_stream s) {
    if (!w || !X || !acts || !pre || !dY || !dW || !db || !work || n <= 0 || n % 16)
        return mfail(SF_EINVAL, "bad argument (n must be a multiple of 16)");
    const long ld = kTile;
    float *G = work, *dA = work + (long)n * ld;
    const float *g_in = dY;   // gradient w.r.t. the current layer's output
    for (int l = SF_MLP_LAYERS - 1; l >= 0; --l) {
        const bool last = l == SF_MLP_LAYERS - 1;
        if (!last) {
            sf::mlp::k_act_back<<<nblk((long)n * ld, 256), 256, 0, S(s)>>>(
                n, g_in, pre + (long)l * n * ld, G, sf::mlp::act_code(w));
        } else {
            const cudaError_t ec = cudaMemcpyAsync(G, g_in, sizeof(float) * n * ld,
                                                   cudaMemcpyDeviceToDevice, S(s));
            if (ec != cudaSuccess) return mcuda(ec, "sf_mlp_backward: copy of dY");
        }
        const float *Xl = l == 0 ? X : acts + (long)(l - 1) * n * ld;
        // dW[out, in] = sum_m G[m, out] Xl[m, in]
        int rc = sf_mlp_gemm(kTile, n, G, 0, 1, ld, Xl, 0, 1, ld, nullptr, 0, dW[l], ld, nullptr, 0,
                             err, s);
        if (rc) return rc;
        const cudaError_t ez = cudaMemsetAsync(db[l], 0, sizeof(float) * kTile, S(s));
        if (ez != cudaSuccess) return mcuda(ez, "sf_mlp_backward: clearing db");
        sf::mlp::k_colsum<<<256, kTile, 0, S(s)>>>(n, G, db[l]);
        if (l > 0) {   // dA[m, in] = sum_out G[m, out] W[out, in]
            rc = sf_mlp_gemm(n, kTile, G, 0, ld, 1, w->W[l], 1, 1, ld, nullptr, 0, dA, ld, nullptr, 0,
                             err, s);
            if (rc) return rc;
            g_in = dA;
            // the next iteration reads dA into G before dA is written again
        }
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_mlp_backward");
}

int sf_mlp_mse(int n, int nvalid, const float *Y, const float *T, float *dY, float *loss, sf_stream s) {
    if (n <= 0 || !Y || !T || !dY || !loss) return mfail(SF_EINVAL, "bad argument");
    sf::mlp::k_mse<<<nblk((long)n * kTile, 256), 256, 0, S(s)>>>(n, nvalid, Y, T, dY, loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_mlp_mse");
}

int sf_mlp_adam(long n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr,
                float b1, float b2, int step, float eps, sf_stream s) {
    if (n <= 0 || !w || !g || !m || !v || step < 1) return mfail(SF_EINVAL, "bad argument");
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    sf::mlp::k_adam<<<nblk(n, 256), 256, 0, S(s)>>>(n, w, g, m, v, (__nv_bfloat16 *)w_bf16, lr, b1, b2,
                                                     c1, c2, eps);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_mlp_adam");
}

int sf_closure_features(sf_ctx *c, const void *u, const void *v, const void *z_r, const void *bvf,
                        const void *sustr, const void *svstr, float *X, sf_stream s) {
    if (!c || !X) return mfail(SF_EINVAL, "bad argument");
    if (2 * (c->N - 1) + 3 > kTile) return mfail(SF_EUNSUPPORTED, "closure rows hold N <= 63 levels");
    cudaError_t e;
    if (c->prec == SF_FP64) {
        auto g = sf::Ops<double>::geo(c);
        sf::mlp::k_features<double><<<nblk(c->s2, 128), 128, 0, S(s)>>>(
            g, (const double *)u, (const double *)v, (const double *)z_r, (const double *)bvf,
            (const double *)sustr, (const double *)svstr, X);
    } else {
        auto g = sf::Ops<float>::geo(c);
        sf::mlp::k_features<float><<<nblk(c->s2, 128), 128, 0, S(s)>>>(
            g, (const float *)u, (const float *)v, (const float *)z_r, (const float *)bvf,
            (const float *)sustr, (const float *)svstr, X);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_closure_features");
}

int sf_closure_apply(sf_ctx *c, const float *Y, const uint8_t *fallback, void *Akv, void *Akt,
                     sf_stream s) {
    if (!c || !Y) return mfail(SF_EINVAL, "bad argument");
    if (2 * (c->N - 1) > kTile) return mfail(SF_EUNSUPPORTED, "closure rows hold N <= 63 levels");
    if (c->prec == SF_FP64) {
        auto g = sf::Ops<double>::geo(c);
        sf::mlp::k_apply<double><<<nblk(c->s2, 128), 128, 0, S(s)>>>(g, Y, fallback, (double *)Akv,
                                                                      (double *)Akt);
    } else {
        auto g = sf::Ops<float>::geo(c);
        sf::mlp::k_apply<float><<<nblk(c->s2, 128), 128, 0, S(s)>>>(g, Y, fallback, (float *)Akv,
                                                                     (float *)Akt);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_closure_apply");
}

int sf_mlp_infer(const sf_mlp_params *w, int n, const float *X, float *Y, int *err, sf_stream s) {
    if (!w || !X || !Y || !err || n < 0) return mfail(SF_EINVAL, "bad argument");
    if (n == 0) return SF_OK;
    sf::mlp::InferW iw;
    for (int l = 0; l < SF_MLP_LAYERS; ++l) {
        if (!w->W[l]) return mfail(SF_EINVAL, "null weight matrix");
        iw.W[l] = static_cast<const __nv_bfloat16 *>(w->W[l]);
        iw.b[l] = w->b[l];
    }
    static bool attr_set[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mcuda(e, "sf_mlp_infer");
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        e = cudaFuncSetAttribute(sf::mlp::k_infer<sf::mlp::kActGelu>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sf::mlp::kInferSmem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(sf::mlp::k_infer<sf::mlp::kActRelu>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sf::mlp::kInferSmem);
        if (e != cudaSuccess) return mcuda(e, "cudaFuncSetAttribute");
        attr_set[dev] = true;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long tiles = ((long)n + kTile - 1) / kTile;
    const unsigned grid = (unsigned)(tiles < sms ? tiles : sms);
    if (w->act == SF_MLP_RELU)
        sf::mlp::k_infer<sf::mlp::kActRelu><<<grid, sf::mlp::kInferThreads, sf::mlp::kInferSmem, S(s)>>>(
            iw, n, X, Y, err);
    else
        sf::mlp::k_infer<sf::mlp::kActGelu><<<grid, sf::mlp::kInferThreads, sf::mlp::kInferSmem, S(s)>>>(
            iw, n, X, Y, err);
    e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_mlp_infer");
}

int sf_closure_step(sf_ctx *c, const sf_mlp_params *w, const void *u, const void *v,
                    const void *z_r, const void *bvf, const void *sustr, const void *svstr,
                    int nfeat, const float *lo, const float *hi, uint8_t *fallback,
                    int *fallback_list, int *fallback_count, void *Akv, void *Akt, int *err,
                    sf_stream s) {
    if (!c || !w || !u || !v || !z_r || !bvf || !sustr || !svstr || !lo || !hi || !fallback ||
        !Akv || !Akt || !err || nfeat < 0 || nfeat > kTile || (!fallback_list != !fallback_count))
        return mfail(SF_EINVAL, "bad argument");
    if (2 * (c->N - 1) + 3 > kTile) return mfail(SF_EUNSUPPORTED, "closure rows hold N <= 63 levels");
    sf::mlp::InferW iw;
    for (int l = 0; l < SF_MLP_LAYERS; ++l) {
        if (!w->W[l]) return mfail(SF_EINVAL, "null weight matrix");
        iw.W[l] = static_cast<const __nv_bfloat16 *>(w->W[l]);
        iw.b[l] = w->b[l];
    }
    const long tiles = (c->s2 + kTile - 1) / kTile;
    const size_t xbytes = (size_t)tiles * kTile * kTile * sizeof(__nv_bfloat16);
    cudaError_t e;
    if (c->closure_x_bytes < xbytes) {   // context-owned scratch: the feature-row tiles
        if (c->closure_x) cudaFree(c->closure_x);
        c->closure_x = nullptr;
        c->closure_x_bytes = 0;
        e = cudaMalloc(&c->closure_x, xbytes);
        if (e != cudaSuccess) return mfail(SF_ENOMEM, "sf_closure_step: feature tiles");
        c->closure_x_bytes = xbytes;
    }
    static bool attr_set[2][64] = {};
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mcuda(e, "sf_closure_step");
    const int pi = c->prec == SF_FP64 ? 1 : 0;
    using sf::mlp::k_closure_mlp;
    using sf::mlp::kActGelu;
    using sf::mlp::kActRelu;
    const bool relu = w->act == SF_MLP_RELU;
    if (dev >= 0 && dev < 64 && !attr_set[pi][dev]) {
        const int sm = (int)sf::mlp::kClosureSmem;
        const auto at = cudaFuncAttributeMaxDynamicSharedMemorySize;
        e = pi ? cudaFuncSetAttribute(k_closure_mlp<double, kActGelu>, at, sm)
               : cudaFuncSetAttribute(k_closure_mlp<float, kActGelu>, at, sm);
        if (e == cudaSuccess)
            e = pi ? cudaFuncSetAttribute(k_closure_mlp<double, kActRelu>, at, sm)
                   : cudaFuncSetAttribute(k_closure_mlp<float, kActRelu>, at, sm);
        if (e != cudaSuccess) return mcuda(e, "cudaFuncSetAttribute");
        attr_set[pi][dev] = true;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)(tiles < sms ? tiles : sms);
    if (fallback_count) {
        e = cudaMemsetAsync(fallback_count, 0, sizeof(int), S(s));
        if (e != cudaSuccess) return mcuda(e, "sf_closure_step");
    }
    auto *X = static_cast<__nv_bfloat16 *>(c->closure_x);
    const long nrows = tiles * kTile;
    if (pi) {
        auto g = sf::Ops<double>::geo(c);
        sf::mlp::k_closure_rows<double><<<nblk(nrows, 128), 128, 0, S(s)>>>(
            g, (const double *)u, (const double *)v, (const double *)z_r, (const double *)bvf,
            (const double *)sustr, (const double *)svstr, nfeat, lo, hi, fallback, fallback_list,
            fallback_count, X, nrows);
        (relu ? k_closure_mlp<double, kActRelu> : k_closure_mlp<double, kActGelu>)
            <<<grid, sf::mlp::kClosureThreads, sf::mlp::kClosureSmem, S(s)>>>(
                g, iw, X, tiles, fallback, (double *)Akv, (double *)Akt, err);
    } else {
        auto g = sf::Ops<float>::geo(c);
        sf::mlp::k_closure_rows<float><<<nblk(nrows, 128), 128, 0, S(s)>>>(
            g, (const float *)u, (const float *)v, (const float *)z_r, (const float *)bvf,
            (const float *)sustr, (const float *)svstr, nfeat, lo, hi, fallback, fallback_list,
            fallback_count, X, nrows);
        (relu ? k_closure_mlp<float, kActRelu> : k_closure_mlp<float, kActGelu>)
            <<<grid, sf::mlp::kClosureThreads, sf::mlp::kClosureSmem, S(s)>>>(
                g, iw, X, tiles, fallback, (float *)Akv, (float *)Akt, err);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_closure_step");
}

int sf_closure_range_mask(sf_ctx *c, const float *X, int nfeat, const float *lo, const float *hi,
                          uint8_t *mask, sf_stream s) {
    if (!c || !X || !lo || !hi || !mask || nfeat < 0 || nfeat > kTile)
        return mfail(SF_EINVAL, "bad argument");
    sf::mlp::k_range_mask<<<nblk(c->s2, 256), 256, 0, S(s)>>>(c->s2, c->I, c->J, nfeat, X, lo, hi,
                                                               mask);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SF_OK : mcuda(e, "sf_closure_range_mask");
}

// ---- allocation-free backward pass ----------------------------------------------------------
// Some callers of this library cannot allocate device memory at the point where they train:
// a host application that owns every device byte through its own pool and forbids other
// allocators, or a training step issued from a latency-critical loop where an allocator call
// (which can synchronise the device or take a process-wide lock) is not allowed.  For them the
// backward pass's scratch lives in this fixed, file-scope device array instead of a caller
// buffer.  Every GPU that loads the library holds it (2 MiB) until the process exits.
constexpr int kStaticMaxRows = 2048;
static __device__ __align__(256) float g_static_work[2 * kStaticMaxRows * SF_MLP_WIDTH];

namespace {
constexpr int kMaxDevices = 64;
float *g_static_work_addr[kMaxDevices] = {};   // device address of g_static_work, per device
}  // namespace

int sf_mlp_backward_static(const sf_mlp_params *w, int n, const float *X, const float *acts,
                           const float *pre, const float *dY, float *const *dW, float *const *db,
                           int *err, sf_stream s) {
    if (n > kStaticMaxRows)
        return mfail(SF_EINVAL, "sf_mlp_backward_static: n exceeds the 2048 rows of its fixed scratch");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mcuda(e, "sf_mlp_backward_static");
    if (dev < 0 || dev >= kMaxDevices) return mfail(SF_EINVAL, "device ordinal out of range");
    if (!g_static_work_addr[dev]) {
        // First call on this device (with it current): the array's name is only a host-side
        // stand-in, so look up its device address once.
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_work);
        if (e != cudaSuccess) return mcuda(e, "cudaGetSymbolAddress");
        g_static_work_addr[dev] = static_cast<float *>(ptr);
    }
    return sf_mlp_backward(w, n, X, acts, pre, dY, dW, db, g_static_work_addr[dev], err, s);
}

}  // extern "C"
