// Learned λ warm start: a 9→64→64→1 MLP (SiLU) predicting each constraint's initial Lagrange multiplier from local
// features. Inference, training (forward, backward) and the Adam update are hand-written kernels; every matrix
// product runs on the sm_100a tcgen05 tensor cores as BF16 operands with FP32 accumulation: 128-row tiles,
// tcgen05.mma issued by one thread on shared-memory operands, accumulators in tensor memory read back with
// tcgen05.ld — inference: layer 1 [128 x 16 (9 padded)] x [16 x 64], layer 2 [128 x 64] x [64 x 64], layer 3 a
// 64-wide dot product; training: the same forward, then dh1 = dz2 · W2 and the weight gradients with the batch rows
// as the reduction dimension. No reference counterpart: the reference has no learned component.
//
// Features of constraint e = (i, j) at the predicted positions of the substep, before any iteration:
//   f0 strain (|xi-xj| - rest)/rest      f1 previous-substep λ · (wi + wj + α̃)/rest
//   f2 ((vi - vj)·n̂)·dt/rest             f3 log10(max(α, 1e-12))          f4 rest length
//   f5..f7 constraint type one-hot         f8 1 if an endpoint is pinned
// f0..f4 are standardised with the dataset's mean/std. The target is t = λ·(wi + wj + α̃)/rest, the multiplier in
// strain units; the network predicts its change over the previous substep, t - f1, standardised — so a network that
// outputs the mean change reproduces the previous-λ warm start, and the learning spends its capacity on the update.
#include <cuda_bf16.h>
#include <mutex>
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_internal.h"
#include "xpbd_kernels.h"
#include "xpbd_tcgen05.h"

namespace xpbd {

namespace {
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
// σ(z) = (1 + tanh(z/2)) / 2 on the hardware tanh approximation (tanh.approx.f32, one instruction): its error (about
// 2^-11 relative to tanh) stays well below the BF16 rounding of the activations that follows, and it replaces an
// exponential and an IEEE division in the SiLU that every hidden unit of every constraint evaluates.
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigm(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = sigm(z);
    return s * (1.0f + z * (1.0f - s));
}

// Raw (unstandardised) features of packed constraint e at the predicted positions jac[0]; `scale` = rest/(wi+wj+α̃).
__device__ __forceinline__ void raw_features(const XpbdWorld& W, const XpbdDevParams& P, uint32_t e, float f[9],
                                             float& scale) {
    const uint4 c = W.con_in[e];
    const float4 pi = W.jac[0][c.x], pj = W.jac[0][c.y];
    const float4 vi = W.v[c.x], vj = W.v[c.y];
    const float rest = __uint_as_float(c.z), comp = __uint_as_float(c.w);
    const float gx = pi.x - pj.x, gy = pi.y - pj.y, gz = pi.z - pj.z;
    const float len = sqrtf(gx * gx + gy * gy + gz * gz);
    const float inv = len > 1e-8f ? 1.0f / len : 0.0f;
    const float alpha_t = comp * P.inv_dt_sq;
    const float denom = pi.w + pj.w + alpha_t;
    const uint32_t ii = W.inc_of_con[2 * e], ij = W.inc_of_con[2 * e + 1];
    const float lam_prev = ii != 0xFFFFFFFFu ? W.inc_lambda[ii] : (ij != 0xFFFFFFFFu ? W.inc_lambda[ij] : 0.0f);
    const float rinv = 1.0f / rest;
    f[0] = (len - rest) * rinv;
    f[1] = lam_prev * denom * rinv;
    f[2] = ((vi.x - vj.x) * gx + (vi.y - vj.y) * gy + (vi.z - vj.z) * gz) * inv * P.dt * rinv;
    f[3] = log10f(fmaxf(comp, 1e-12f));
    f[4] = rest;
    const uint32_t ty = W.con_type[e];
    f[5] = ty == 0 ? 1.0f : 0.0f;
    f[6] = ty == 1 ? 1.0f : 0.0f;
    f[7] = ty == 2 ? 1.0f : 0.0f;
    f[8] = (pi.w <= 0.0f || pj.w <= 0.0f) ? 1.0f : 0.0f;
    scale = denom > 0.0f ? rest / denom : 0.0f;
}
}  // namespace

// ---- inference on the tcgen05 tensor cores: 128 constraints per tile, one thread per row.
// Layer 1 (M=128, N=64, K=16) and layer 2 (M=128, N=64, K=64, four K steps) are tcgen05.mma instructions issued by
// one thread on BF16 operands in shared memory, accumulating in FP32 in tensor memory (columns 0-63 and 64-127);
// each thread reads its row's accumulators back with tcgen05.ld, adds the bias, applies SiLU, and either stores the
// BF16 activations as the next layer's A operand or forms the output dot product. The rounding points are those of
// the training forward: BF16 inputs, weights and hidden activations, FP32 accumulation and output.
struct TcSmem {
    __nv_bfloat16 w1[64 * 16];   // B of layer 1, canonical K-major layout (see tc_index)
    __nv_bfloat16 w2[64 * 64];   // B of layer 2
    __nv_bfloat16 a1[128 * 16];  // A of layer 1: the tile's standardised features
    __nv_bfloat16 a2[128 * 64];  // A of layer 2: the tile's BF16 hidden activations
    float b1[64], b2[64], w3[64];
    float fmean[XPBD_MLP_IN], fstd[XPBD_MLP_IN], b3, tmean, tstd;
    uint64_t bar;
    uint32_t tmem;
};
// Dynamic shared memory per CTA: padded so that at most four CTAs share an SM (4 × 128 = its 512 tensor-memory
// columns), so the allocation never waits.
constexpr size_t kTcSmemBytes = 50 * 1024;
constexpr uint32_t kTcCtasPerSm = 4;
constexpr uint32_t kTcCols = 128;
constexpr uint32_t kTcIdesc = tc_idesc_bf16(128, 64);

// Element index of (row r, column k) of an R-row K-major BF16 matrix in the no-swizzle canonical layout: 8-element
// K chunks are planes of R × 16 bytes (lbo = 16·R); inside a plane, 8-row groups of 128 bytes (sbo = 128).
__device__ __forceinline__ uint32_t tc_index(uint32_t r, uint32_t k, uint32_t rows) {
    return (((k >> 3) * (rows >> 3) + (r >> 3)) * 8u + (r & 7u)) * 8u + (k & 7u);
}

__device__ void tc_load_mlp(TcSmem& s, const XpbdMlp& m) {
    const __nv_bfloat16* w1 = reinterpret_cast<const __nv_bfloat16*>(m.w1);
    const __nv_bfloat16* w2 = reinterpret_cast<const __nv_bfloat16*>(m.w2);
    for (uint32_t q = threadIdx.x; q < 64 * 16; q += blockDim.x) s.w1[tc_index(q >> 4, q & 15u, 64)] = w1[q];
    for (uint32_t q = threadIdx.x; q < 64 * 64; q += blockDim.x) s.w2[tc_index(q >> 6, q & 63u, 64)] = w2[q];
    for (uint32_t k = threadIdx.x; k < 64; k += blockDim.x) {
        s.b1[k] = m.b1[k];
        s.b2[k] = m.b2[k];
        s.w3[k] = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(m.w3)[k]);
    }
    if (threadIdx.x < XPBD_MLP_IN) {
        s.fmean[threadIdx.x] = m.fmean[threadIdx.x];
        s.fstd[threadIdx.x] = m.fstd[threadIdx.x];
    }
    if (threadIdx.x == 0) {
        s.b3 = m.b3;
        s.tmean = m.tmean;
        s.tstd = m.tstd;
    }
}

// This thread's row of the layer-1 operand: standardised features, BF16, columns 9..15 zero.
__device__ __forceinline__ void tc_store_features(TcSmem& s, uint32_t r, const float f[9]) {
    __nv_bfloat16 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k)
        v[k] = __float2bfloat16_rn(k < 5 ? (f[k] - s.fmean[k]) / s.fstd[k] : (k < 9 ? f[k] : 0.0f));
    *reinterpret_cast<uint4*>(s.a1 + tc_index(r, 0, 128)) = *reinterpret_cast<const uint4*>(v);
    *reinterpret_cast<uint4*>(s.a1 + tc_index(r, 8, 128)) = *reinterpret_cast<const uint4*>(v + 8);
}
// Forward of the tile whose layer-1 operand is staged (every thread called tc_store_features): returns this
// thread's row output y (standardised). `phase` is the mbarrier parity of the next completion; false when a wait gave
// up (the kernel then stops).
__device__ __forceinline__ bool tc_tile_forward(TcSmem& s, uint32_t& phase, float& y) {
    const uint32_t r = threadIdx.x, warp = r >> 5;
    const uint32_t lane_base = s.tmem + ((32u * warp) << 16);
    tc_fence_proxy();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (r == 0) {
        tc_mma(s.tmem, tc_desc(tc_smem_addr(s.a1), 128 * 16, 128), tc_desc(tc_smem_addr(s.w1), 64 * 16, 128),
               kTcIdesc, false);
        tc_commit(&s.bar);
    }
    bool ok = tc_mbar_wait(&s.bar, phase);
    phase ^= 1u;
    tc_fence_after();
    // layer-1 epilogue: bias, SiLU, BF16 → this row of the layer-2 operand
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float z[16];
        tc_ld16(lane_base + 16u * c, z);
        __nv_bfloat16 h[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) h[k] = __float2bfloat16_rn(silu(z[k] + s.b1[16 * c + k]));
        *reinterpret_cast<uint4*>(s.a2 + tc_index(r, 16 * c, 128)) = *reinterpret_cast<const uint4*>(h);
        *reinterpret_cast<uint4*>(s.a2 + tc_index(r, 16 * c + 8, 128)) = *reinterpret_cast<const uint4*>(h + 8);
    }
    tc_fence_proxy();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (r == 0) {
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q)  // K steps of 16: two 8-element chunk planes each
            tc_mma(s.tmem + 64u, tc_desc(tc_smem_addr(s.a2) + q * 2u * 128u * 16u, 128 * 16, 128),
                   tc_desc(tc_smem_addr(s.w2) + q * 2u * 64u * 16u, 64 * 16, 128), kTcIdesc, q > 0);
        tc_commit(&s.bar);
    }
    ok = tc_mbar_wait(&s.bar, phase) && ok;
    phase ^= 1u;
    tc_fence_after();
    float acc = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float z[16];
        tc_ld16(lane_base + 64u + 16u * c, z);
#pragma unroll
        for (int k = 0; k < 16; ++k) acc += bf16r(silu(z[k] + s.b2[16 * c + k])) * s.w3[16 * c + k];
    }
    y = acc + s.b3;
    // every thread's reads of the accumulators and of the operands end before the next tile overwrites them; the
    // verdict of the waits is made uniform so that every thread leaves the tile loop together
    tc_fence_before();
    return __syncthreads_and(ok) != 0;
}

__device__ __forceinline__ void tc_setup(TcSmem& s, const XpbdMlp& m) {
    tc_load_mlp(s, m);
    if (threadIdx.x == 0) tc_mbar_init(&s.bar, 1);
    if (threadIdx.x < 32) tc_alloc(&s.tmem, kTcCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}
__device__ __forceinline__ void tc_teardown(TcSmem& s) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32) tc_dealloc(s.tmem, kTcCols);
}

// ---- inference: λ0 for every constraint, written to both incidences (warm_lam_inc)
__global__ void __launch_bounds__(128) mlp_infer_kernel(XpbdWorld W, const XpbdMlp* __restrict__ mlp) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
    tc_setup(S, *mlp);
    const XpbdDevParams P = *W.params;
    uint32_t phase = 0;
    const uint32_t tiles = (W.e + 127) / 128;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t e = tile * 128 + threadIdx.x;
        float f[9], scale = 0.0f;
        if (e < W.e) {
            raw_features(W, P, e, f, scale);
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) f[k] = 0.0f;
        }
        tc_store_features(S, threadIdx.x, f);
        float y;
        if (!tc_tile_forward(S, phase, y)) {
            if (threadIdx.x == 0) atomicOr(W.status, XPBD_DEV_BARRIER_TIMEOUT);
            break;
        }
        if (e < W.e) {
            const float lam = (y * S.tstd + S.tmean + f[1]) * scale;
            const uint32_t a = W.inc_of_con[2 * e], b = W.inc_of_con[2 * e + 1];
            if (a != 0xFFFFFFFFu) W.warm_lam_inc[a] = lam;
            if (b != 0xFFFFFFFFu) W.warm_lam_inc[b] = lam;
        }
    }
    tc_teardown(S);
}

// ---- inference on given raw features (tests): out[r] = standardised prediction y
__global__ void __launch_bounds__(128) mlp_eval_kernel(const XpbdMlp* __restrict__ mlp, const float* __restrict__ feat,
                                                       uint32_t n, float* __restrict__ out) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& S = *reinterpret_cast<TcSmem*>(tc_raw);
    tc_setup(S, *mlp);
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x; tile < (n + 127) / 128; tile += gridDim.x) {
        const uint32_t r = tile * 128 + threadIdx.x;
        float f[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = r < n ? feat[(size_t)r * 9 + k] : 0.0f;
        tc_store_features(S, threadIdx.x, f);
        float y;
        if (!tc_tile_forward(S, phase, y)) break;
        if (r < n) out[r] = y;
    }
    tc_teardown(S);
}

// ---- dataset collection: sampled constraints e = offset + m*stride
__global__ void mlp_collect_features_kernel(XpbdWorld W, uint32_t stride, uint32_t offset, float* __restrict__ feat,
                                            float* __restrict__ scale, uint32_t base, uint32_t cap) {
    const XpbdDevParams P = *W.params;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;; m += gridDim.x * blockDim.x) {
        const uint64_t e = (uint64_t)offset + (uint64_t)m * stride;
        if (e >= W.e || base + m >= cap) break;
        float f[9], sc;
        raw_features(W, P, (uint32_t)e, f, sc);
        for (int k = 0; k < 9; ++k) feat[(size_t)(base + m) * 9 + k] = f[k];
        scale[base + m] = sc;
    }
}
__global__ void mlp_collect_targets_kernel(XpbdWorld W, uint32_t stride, uint32_t offset, const float* __restrict__ scale,
                                           float* __restrict__ target, uint32_t base, uint32_t cap) {
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x;; m += gridDim.x * blockDim.x) {
        const uint64_t e = (uint64_t)offset + (uint64_t)m * stride;
        if (e >= W.e || base + m >= cap) break;
        const uint32_t ii = W.inc_of_con[2 * e], ij = W.inc_of_con[2 * e + 1];
        const float lam = ii != 0xFFFFFFFFu ? W.inc_lambda[ii] : (ij != 0xFFFFFFFFu ? W.inc_lambda[ij] : 0.0f);
        const float sc = scale[base + m];
        target[base + m] = sc > 0.0f ? lam / sc : 0.0f;
    }
}

// ---- training: gradients of mean((y - (t - f1 - tmean)/tstd)^2) over the rows listed in idx
// grads layout (fp32): w1[64][9], b1[64], w2[64][64], b2[64], w3[64], b3; loss (sum of squares) at loss[0].
// ---- Adam on the fp32 master parameters, then the bf16 working copy
__global__ void mlp_adam_kernel(float* __restrict__ master, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ grads, float gscale, float lr, float beta1, float beta2,
                                float eps, float bc1, float bc2, XpbdMlp* __restrict__ mlp) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < XPBD_MLP_PARAMS; k += gridDim.x * blockDim.x) {
        const float gk = grads[k] * gscale;
        const float a = beta1 * m1[k] + (1.0f - beta1) * gk;
        const float b = beta2 * m2[k] + (1.0f - beta2) * gk * gk;
        m1[k] = a;
        m2[k] = b;
        const float p = master[k] - lr * (a / bc1) / (sqrtf(b / bc2) + eps);
        master[k] = p;
    }
}

// master (fp32, flat) → working copy (bf16 weights [out][in], padded) + fp32 biases
__global__ void mlp_publish_kernel(const float* __restrict__ master, XpbdMlp* __restrict__ mlp) {
    __nv_bfloat16* w1 = reinterpret_cast<__nv_bfloat16*>(mlp->w1);
    __nv_bfloat16* w2 = reinterpret_cast<__nv_bfloat16*>(mlp->w2);
    __nv_bfloat16* w3 = reinterpret_cast<__nv_bfloat16*>(mlp->w3);
    for (uint32_t k = threadIdx.x; k < 64 * 16; k += blockDim.x) {
        const uint32_t o = k / 16, i = k % 16;
        w1[k] = __float2bfloat16_rn(i < 9 ? master[o * 9 + i] : 0.0f);
    }
    for (uint32_t k = threadIdx.x; k < 64; k += blockDim.x) {
        mlp->b1[k] = master[576 + k];
        mlp->b2[k] = master[576 + 64 + 4096 + k];
        w3[k] = __float2bfloat16_rn(master[576 + 64 + 4096 + 64 + k]);
    }
    for (uint32_t k = threadIdx.x; k < 64 * 64; k += blockDim.x) w2[k] = __float2bfloat16_rn(master[576 + 64 + k]);
    if (threadIdx.x == 0) mlp->b3 = master[XPBD_MLP_PARAMS - 1];
}

// ---- training step on the tcgen05 tensor cores: 128 sampled rows per tile, one thread per row.
// Forward as in inference (layer 1: M 128, N 64, K 16; layer 2: K 64), then the backward products, each one
// tcgen05.mma chain on K-major BF16 operands in shared memory with FP32 accumulation in tensor memory:
//   dh1 = dz2 · W2         M 128 rows,  N 64 (in),  K 64 (out)   A = dz2, B = W2ᵀ (a transposed copy)
//   dW2 += dz2ᵀ · h1       M 128 (out in rows 0..63), N 64 (in), K 128 rows   A = dz2ᵀ, B = h1ᵀ
//   dW1 += dz1ᵀ · x        M 128 (out in rows 0..63), N 16 (features), K 128 rows   A = dz1ᵀ, B = xᵀ
// (rows 64..127 of those A operands are never written: they only produce accumulator rows 64..127, never read)
// The epilogues write each row's values both row-major and transposed (the transposed copies are the K-major
// operands of the weight gradients), and dW2 and dW1 accumulate in tensor memory over all the CTA's tiles. The
// rounding points are those of the forward and of the reference-checked gradient: BF16 operands (x, h1, dz2, dz1,
// weights), FP32 accumulation, FP32 bias and output-layer gradients. Tensor-memory columns: z1 0-63, z2 then dh1
// 64-127, dW2 128-191, dW1 192-207.
struct TcTrainSmem {
    __nv_bfloat16 w1[64 * 16];     // B of layer 1
    __nv_bfloat16 w2[64 * 64];     // B of layer 2: [out][in]
    __nv_bfloat16 w2t[64 * 64];    // B of dh1: [in][out]
    __nv_bfloat16 a1[128 * 16];    // x  (A of layer 1)
    __nv_bfloat16 xt[16 * 128];    // xᵀ (B of dW1)
    __nv_bfloat16 a2[128 * 64];    // h1 (A of layer 2)
    __nv_bfloat16 h1t[64 * 128];   // h1ᵀ (B of dW2)
    __nv_bfloat16 dz2[128 * 64];   // dz2 (A of dh1)
    __nv_bfloat16 dz2t[128 * 128]; // dz2ᵀ (A of dW2; rows 64..127 unwritten: they only reach D rows never read)
    __nv_bfloat16 dz1t[128 * 128]; // dz1ᵀ (A of dW1; the same)
    float b1[64], b2[64], w3[64];
    float fmean[XPBD_MLP_IN], fstd[XPBD_MLP_IN], b3, tmean, tstd;
    float gb1[64], gb2[64], gw3[64], gb3, loss;
    uint64_t bar;
    uint32_t tmem;
};
constexpr size_t kTcTrainSmemBytes = (sizeof(TcTrainSmem) + 1023) / 1024 * 1024;
constexpr uint32_t kTcTrainCols = 256;

// Sum over the warp's 32 rows of v; lane 0 adds it to *dst (shared memory).
__device__ __forceinline__ void warp_sum_to(float v, float* dst) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(dst, v);
}

// One MMA chain issued by thread 0 and completed through the mbarrier: D (+)= A·Bᵀ over `ksteps` K-steps of 16;
// `ra` / `rb` are the rows (M / N) of the K-major A and B tiles.
__device__ __forceinline__ void tc_chain(uint32_t tmem_d, const __nv_bfloat16* a, uint32_t ra, const __nv_bfloat16* b,
                                         uint32_t rb, uint32_t ksteps, uint32_t idesc, bool accumulate) {
    for (uint32_t q = 0; q < ksteps; ++q)
        tc_mma(tmem_d, tc_desc(tc_smem_addr(a) + q * 2u * ra * 16u, ra * 16u, 128u),
               tc_desc(tc_smem_addr(b) + q * 2u * rb * 16u, rb * 16u, 128u), idesc, accumulate || q > 0);
}

__global__ void __launch_bounds__(128) mlp_train_tc_kernel(const XpbdMlp* __restrict__ mlp,
                                                           const float* __restrict__ feat,
                                                           const float* __restrict__ target,
                                                           const uint32_t* __restrict__ idx, uint32_t nrows,
                                                           float* __restrict__ grads, float* __restrict__ loss,
                                                           int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char tt_raw[];
    TcTrainSmem& T = *reinterpret_cast<TcTrainSmem*>(tt_raw);
    const uint32_t r = threadIdx.x, warp = r >> 5;
    const __nv_bfloat16* w1 = reinterpret_cast<const __nv_bfloat16*>(mlp->w1);
    const __nv_bfloat16* w2 = reinterpret_cast<const __nv_bfloat16*>(mlp->w2);
    for (uint32_t q = r; q < 64 * 16; q += blockDim.x) T.w1[tc_index(q >> 4, q & 15u, 64)] = w1[q];
    for (uint32_t q = r; q < 64 * 64; q += blockDim.x) {
        const uint32_t o = q >> 6, i = q & 63u;
        T.w2[tc_index(o, i, 64)] = w2[q];
        T.w2t[tc_index(i, o, 64)] = w2[q];
    }
    for (uint32_t k = r; k < 64; k += blockDim.x) {
        T.b1[k] = mlp->b1[k];
        T.b2[k] = mlp->b2[k];
        T.w3[k] = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(mlp->w3)[k]);
        T.gb1[k] = T.gb2[k] = T.gw3[k] = 0.0f;
    }
    if (r < XPBD_MLP_IN) {
        T.fmean[r] = mlp->fmean[r];
        T.fstd[r] = mlp->fstd[r];
    }
    if (r == 0) {
        T.b3 = mlp->b3;
        T.tmean = mlp->tmean;
        T.tstd = mlp->tstd;
        T.gb3 = 0.0f;
        T.loss = 0.0f;
        tc_mbar_init(&T.bar, 1);
    }
    if (warp == 0) tc_alloc(&T.tmem, kTcTrainCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t lane_base = T.tmem + ((32u * warp) << 16);
    constexpr uint32_t kId64 = tc_idesc_bf16(128, 64), kId16 = tc_idesc_bf16(128, 16);
    const float inv_b = 1.0f / (float)nrows;
    const uint32_t tiles = (nrows + 127) / 128;
    uint32_t phase = 0;
    bool ok = true, first = true;
    float loss_acc = 0.0f;
    auto issue_and_wait = [&](auto&& issue) {
        tc_fence_proxy();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (r == 0) {
            issue();
            tc_commit(&T.bar);
        }
        ok = tc_mbar_wait(&T.bar, phase) && ok;
        phase ^= 1u;
        tc_fence_after();
    };
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t row = tile * 128 + r;
        const bool valid = row < nrows;
        const uint32_t sample = valid ? idx[row] : 0u;
        float f[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) f[k] = valid ? feat[(size_t)sample * 9 + k] : 0.0f;
        const float tgt = valid ? (target[sample] - f[1] - T.tmean) / T.tstd : 0.0f;
        {  // x: standardised features, BF16, row-major (layer 1) and transposed (dW1)
            __nv_bfloat16 xv[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                xv[k] = __float2bfloat16_rn(k < 5 ? (f[k] - T.fmean[k]) / T.fstd[k] : (k < 9 ? f[k] : 0.0f));
                T.xt[tc_index(k, r, 16)] = xv[k];
            }
            *reinterpret_cast<uint4*>(T.a1 + tc_index(r, 0, 128)) = *reinterpret_cast<const uint4*>(xv);
            *reinterpret_cast<uint4*>(T.a1 + tc_index(r, 8, 128)) = *reinterpret_cast<const uint4*>(xv + 8);
        }
        issue_and_wait([&] { tc_chain(T.tmem, T.a1, 128, T.w1, 64, 1, kId64, false); });
        // h1 = BF16(SiLU(z1 + b1)): row-major (layer 2) and transposed (dW2)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float z[16];
            tc_ld16(lane_base + 16u * c, z);
            __nv_bfloat16 h[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                h[k] = __float2bfloat16_rn(silu(z[k] + T.b1[16 * c + k]));
                T.h1t[tc_index(16 * c + k, r, 64)] = h[k];
            }
            *reinterpret_cast<uint4*>(T.a2 + tc_index(r, 16 * c, 128)) = *reinterpret_cast<const uint4*>(h);
            *reinterpret_cast<uint4*>(T.a2 + tc_index(r, 16 * c + 8, 128)) = *reinterpret_cast<const uint4*>(h + 8);
        }
        issue_and_wait([&] { tc_chain(T.tmem + 64u, T.a2, 128, T.w2, 64, 4, kId64, false); });
        // output, error and dz2 = dy · w3 · SiLU'(z2 + b2) (two reads of z2: dy needs the whole row first)
        float y = 0.0f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            float z[16];
            tc_ld16(lane_base + 64u + 16u * c, z);
#pragma unroll
            for (int k = 0; k < 16; ++k) y += bf16r(silu(z[k] + T.b2[16 * c + k])) * T.w3[16 * c + k];
        }
        y += T.b3;
        const float e = valid ? y - tgt : 0.0f;
        loss_acc += e * e;
        const float dy = 2.0f * e * inv_b;
        warp_sum_to(dy, &T.gb3);
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float z[16];
            tc_ld16(lane_base + 64u + 16u * c, z);
            __nv_bfloat16 d[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int u = 16 * c + k;
                const float zz = z[k] + T.b2[u];
                warp_sum_to(dy * bf16r(silu(zz)), &T.gw3[u]);
                const float dz = dy * T.w3[u] * dsilu(zz);
                warp_sum_to(dz, &T.gb2[u]);
                d[k] = __float2bfloat16_rn(dz);
                T.dz2t[tc_index(u, r, 128)] = d[k];
            }
            *reinterpret_cast<uint4*>(T.dz2 + tc_index(r, 16 * c, 128)) = *reinterpret_cast<const uint4*>(d);
            *reinterpret_cast<uint4*>(T.dz2 + tc_index(r, 16 * c + 8, 128)) = *reinterpret_cast<const uint4*>(d + 8);
        }
        const bool acc = !first;
        issue_and_wait([&] {
            tc_chain(T.tmem + 64u, T.dz2, 128, T.w2t, 64, 4, kId64, false);  // dh1 (over z2's columns)
            tc_chain(T.tmem + 128u, T.dz2t, 128, T.h1t, 64, 8, kId64, acc);  // dW2
        });
        // dz1 = dh1 · SiLU'(z1 + b1), transposed (dW1)
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float dh[16], z[16];
            tc_ld16(lane_base + 64u + 16u * c, dh);
            tc_ld16(lane_base + 16u * c, z);
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const int u = 16 * c + k;
                const float dz = dh[k] * dsilu(z[k] + T.b1[u]);
                warp_sum_to(dz, &T.gb1[u]);
                T.dz1t[tc_index(u, r, 128)] = __float2bfloat16_rn(dz);
            }
        }
        issue_and_wait([&] { tc_chain(T.tmem + 192u, T.dz1t, 128, T.xt, 16, 8, kId16, acc); });
        first = false;
        // every MMA of this tile has completed: the next tile may overwrite the operands
        tc_fence_before();
        if (!__syncthreads_and(ok)) break;
        tc_fence_after();
    }
    warp_sum_to(loss_acc, &T.loss);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!first && warp < 2) {  // dW2 and dW1: tensor-memory lanes 0..63 are the 64 hidden units
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float g[16];
            tc_ld16(lane_base + 128u + 16u * c, g);
#pragma unroll
            for (int k = 0; k < 16; ++k) atomicAdd(&grads[576 + 64 + r * 64 + 16 * c + k], g[k]);
        }
        float g1[16];
        tc_ld16(lane_base + 192u, g1);
#pragma unroll
        for (int k = 0; k < 9; ++k) atomicAdd(&grads[r * 9 + k], g1[k]);
    }
    for (uint32_t k = r; k < 64; k += blockDim.x) {
        atomicAdd(&grads[576 + k], T.gb1[k]);
        atomicAdd(&grads[576 + 64 + 4096 + k], T.gb2[k]);
        atomicAdd(&grads[576 + 64 + 4096 + 64 + k], T.gw3[k]);
    }
    if (r == 0) {
        atomicAdd(&grads[XPBD_MLP_PARAMS - 1], T.gb3);
        atomicAdd(loss, T.loss);
        if (!ok) atomicOr(status, XPBD_DEV_BARRIER_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tc_dealloc(T.tmem, kTcTrainCols);
}

// ---------------------------------------------------------------------------------------------- launchers
static cudaError_t tc_prepare(const void* fn) {
    static_assert(sizeof(TcSmem) <= kTcSmemBytes, "tensor-core MLP shared memory");
    static std::once_flag once;
    static cudaError_t result = cudaSuccess;
    std::call_once(once, [] {
        result = cudaFuncSetAttribute((const void*)mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)kTcSmemBytes);
        if (result == cudaSuccess)
            result = cudaFuncSetAttribute((const void*)mlp_eval_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)kTcSmemBytes);
    });
    (void)fn;
    return result;
}
cudaError_t launch_mlp_infer(const XpbdWorld& W, const XpbdMlp* mlp, int sms, cudaStream_t st) {
    cudaError_t e = tc_prepare((const void*)mlp_infer_kernel);
    if (e != cudaSuccess) return e;
    uint32_t grid = (W.e + 127) / 128;
    if (grid > (uint32_t)sms * kTcCtasPerSm) grid = (uint32_t)sms * kTcCtasPerSm;
    if (grid == 0) grid = 1;
    mlp_infer_kernel<<<grid, 128, kTcSmemBytes, st>>>(W, mlp);
    return cudaGetLastError();
}
cudaError_t launch_mlp_eval(const XpbdMlp* mlp, const float* feat, uint32_t n, float* out, cudaStream_t st) {
    cudaError_t e = tc_prepare((const void*)mlp_eval_kernel);
    if (e != cudaSuccess) return e;
    uint32_t grid = (n + 127) / 128;
    if (grid == 0) grid = 1;
    if (grid > 148 * kTcCtasPerSm) grid = 148 * kTcCtasPerSm;
    mlp_eval_kernel<<<grid, 128, kTcSmemBytes, st>>>(mlp, feat, n, out);
    return cudaGetLastError();
}
cudaError_t launch_mlp_collect_features(const XpbdWorld& W, uint32_t stride, uint32_t offset, float* feat,
                                        float* scale, uint32_t base, uint32_t cap, cudaStream_t st) {
    mlp_collect_features_kernel<<<148, 256, 0, st>>>(W, stride, offset, feat, scale, base, cap);
    return cudaGetLastError();
}
cudaError_t launch_mlp_collect_targets(const XpbdWorld& W, uint32_t stride, uint32_t offset, const float* scale,
                                       float* target, uint32_t base, uint32_t cap, cudaStream_t st) {
    mlp_collect_targets_kernel<<<148, 256, 0, st>>>(W, stride, offset, scale, target, base, cap);
    return cudaGetLastError();
}
cudaError_t launch_mlp_train(const XpbdMlp* mlp, const float* feat, const float* target, const uint32_t* idx,
                             uint32_t nrows, float* grads, float* loss, int* status, cudaStream_t st) {
    // the attribute is per device; setting it again is cheap and idempotent
    static_assert(sizeof(TcTrainSmem) <= kTcTrainSmemBytes, "tensor-core training shared memory");
    if (cudaFuncSetAttribute(mlp_train_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kTcTrainSmemBytes) != cudaSuccess)
        return cudaErrorInvalidValue;
    uint32_t grid = (nrows + 127) / 128;  // one 128-row tile per CTA; one CTA per SM (shared memory)
    if (grid > 148) grid = 148;
    if (grid == 0) grid = 1;
    mlp_train_tc_kernel<<<grid, 128, kTcTrainSmemBytes, st>>>(mlp, feat, target, idx, nrows, grads, loss, status);
    return cudaGetLastError();
}
cudaError_t launch_mlp_adam(float* master, float* m1, float* m2, const float* grads, float gscale, float lr,
                            float beta1, float beta2, float eps, float bc1, float bc2, XpbdMlp* mlp, cudaStream_t st) {
    mlp_adam_kernel<<<20, 256, 0, st>>>(master, m1, m2, grads, gscale, lr, beta1, beta2, eps, bc1, bc2, mlp);
    mlp_publish_kernel<<<1, 256, 0, st>>>(master, mlp);
    return cudaGetLastError();
}
cudaError_t launch_mlp_publish(const float* master, XpbdMlp* mlp, cudaStream_t st) {
    mlp_publish_kernel<<<1, 256, 0, st>>>(master, mlp);
    return cudaGetLastError();
}

}  // namespace xpbd
