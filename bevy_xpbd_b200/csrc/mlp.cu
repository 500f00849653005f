// Learned λ warm start: a 9→64→64→1 MLP (SiLU) predicting each constraint's initial Lagrange multiplier from local
// features. Inference, training (forward, backward) and the Adam update are hand-written kernels; every matrix
// product runs on the tensor cores as BF16 tiles with FP32 accumulation. Inference uses the sm_100a tcgen05 path:
// 128-constraint tiles, tcgen05.mma issued by one thread on shared-memory operands, accumulators in tensor memory
// read back with tcgen05.ld. Training uses warp-level mma.sync.m16n8k16 tiles of 16 constraints (its backward keeps
// the forward's accumulators in registers): layer 1 = [16 x 16(9 padded)] x [16 x 64], layer 2 = [16 x 64] x
// [64 x 64] (the layer-1 accumulator registers are repacked as layer-2 A fragments), layer 3 a 64-wide dot product;
// weight gradients are the same tiles with the batch as the reduction dimension. No reference counterpart: the reference has no learned component.
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
constexpr unsigned kAll = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint32_t two(const __nv_bfloat16 a, const __nv_bfloat16 b) {
    __nv_bfloat162 v;
    v.x = a;
    v.y = b;
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ void mma16816(float* d, const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
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

// Shared-memory copy of the working weights (bf16, [out][in]) and biases.
struct SmemMlp {
    __nv_bfloat16 w1[64 * 16];
    __nv_bfloat16 w2[64 * 64];
    __nv_bfloat16 w3[64];
    float b1[64], b2[64], b3;
    float fmean[XPBD_MLP_IN], fstd[XPBD_MLP_IN], tmean, tstd;
};
__device__ void load_mlp(SmemMlp& s, const XpbdMlp& m) {
    const __nv_bfloat16* w1 = reinterpret_cast<const __nv_bfloat16*>(m.w1);
    const __nv_bfloat16* w2 = reinterpret_cast<const __nv_bfloat16*>(m.w2);
    const __nv_bfloat16* w3 = reinterpret_cast<const __nv_bfloat16*>(m.w3);
    for (uint32_t k = threadIdx.x; k < 64 * 16; k += blockDim.x) s.w1[k] = w1[k];
    for (uint32_t k = threadIdx.x; k < 64 * 64; k += blockDim.x) s.w2[k] = w2[k];
    for (uint32_t k = threadIdx.x; k < 64; k += blockDim.x) {
        s.w3[k] = w3[k];
        s.b1[k] = m.b1[k];
        s.b2[k] = m.b2[k];
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

// Forward of one 16-row tile. xs: the tile's standardised features [16][16] (bf16). Keeps z1, z2 (pre-activations,
// fp32, accumulator layout: per n-tile j the thread holds rows g and g+8, cols 8j+2t, 8j+2t+1) and the bf16 h2 values
// for the backward pass; returns y for rows g (y_lo) and g+8 (y_hi) in every lane of the row's quad.
struct TileFwd {
    float z1[8][4], z2[8][4];
    float y_lo, y_hi;
};
__device__ __forceinline__ void tile_forward(const SmemMlp& S, const __nv_bfloat16* xs, TileFwd& F) {
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 2, t = lane & 3u;
    uint32_t a[4];
    a[0] = ld_pair(xs + g * 16 + 2 * t);
    a[1] = ld_pair(xs + (g + 8) * 16 + 2 * t);
    a[2] = ld_pair(xs + g * 16 + 8 + 2 * t);
    a[3] = ld_pair(xs + (g + 8) * 16 + 8 + 2 * t);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float* d = F.z1[j];
        d[0] = d[1] = d[2] = d[3] = 0.0f;
        const __nv_bfloat16* wb = S.w1 + (8 * j + g) * 16;
        mma16816(d, a, ld_pair(wb + 2 * t), ld_pair(wb + 8 + 2 * t));
        const float b0 = S.b1[8 * j + 2 * t], b1 = S.b1[8 * j + 2 * t + 1];
        d[0] += b0;
        d[1] += b1;
        d[2] += b0;
        d[3] += b1;
    }
    uint32_t a2[4][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const float* c0 = F.z1[2 * kk];
        const float* c1 = F.z1[2 * kk + 1];
        a2[kk][0] = pack_bf16(silu(c0[0]), silu(c0[1]));
        a2[kk][1] = pack_bf16(silu(c0[2]), silu(c0[3]));
        a2[kk][2] = pack_bf16(silu(c1[0]), silu(c1[1]));
        a2[kk][3] = pack_bf16(silu(c1[2]), silu(c1[3]));
    }
    float ylo = 0.0f, yhi = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float* d = F.z2[j];
        d[0] = d[1] = d[2] = d[3] = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const __nv_bfloat16* wb = S.w2 + (8 * j + g) * 64 + 16 * kk;
            mma16816(d, a2[kk], ld_pair(wb + 2 * t), ld_pair(wb + 8 + 2 * t));
        }
        const int c = 8 * j + 2 * t;
        d[0] += S.b2[c];
        d[1] += S.b2[c + 1];
        d[2] += S.b2[c];
        d[3] += S.b2[c + 1];
        const float w3a = __bfloat162float(S.w3[c]), w3b = __bfloat162float(S.w3[c + 1]);
        ylo += bf16r(silu(d[0])) * w3a + bf16r(silu(d[1])) * w3b;
        yhi += bf16r(silu(d[2])) * w3a + bf16r(silu(d[3])) * w3b;
    }
    ylo += __shfl_xor_sync(kAll, ylo, 1);
    ylo += __shfl_xor_sync(kAll, ylo, 2);
    yhi += __shfl_xor_sync(kAll, yhi, 1);
    yhi += __shfl_xor_sync(kAll, yhi, 2);
    F.y_lo = ylo + S.b3;
    F.y_hi = yhi + S.b3;
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
__device__ __forceinline__ void store_row(const SmemMlp& S, const float f[9], __nv_bfloat16* row) {
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const float v = k < 5 ? (f[k] - S.fmean[k]) / S.fstd[k] : f[k];
        row[k] = __float2bfloat16_rn(v);
    }
#pragma unroll
    for (int k = 9; k < 16; ++k) row[k] = __float2bfloat16_rn(0.0f);
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
struct TrainSmem {
    SmemMlp S;
    __nv_bfloat16 xs[4][16 * 16];
    __nv_bfloat16 hs[4][16 * 64];   // h1 (bf16)
    __nv_bfloat16 ds[4][16 * 64];   // dz2, then dz1 (bf16)
    float gw1[64 * 16], gw2[64 * 64], gb1[64], gb2[64], gw3[64], gb3;
};

__global__ void __launch_bounds__(128) mlp_train_kernel(const XpbdMlp* __restrict__ mlp, const float* __restrict__ feat,
                                                        const float* __restrict__ target,
                                                        const uint32_t* __restrict__ idx, uint32_t nrows,
                                                        float* __restrict__ grads, float* __restrict__ loss) {
    extern __shared__ __align__(16) unsigned char t_smem[];
    TrainSmem& T = *reinterpret_cast<TrainSmem*>(t_smem);
    load_mlp(T.S, *mlp);
    for (uint32_t k = threadIdx.x; k < 64 * 16; k += blockDim.x) T.gw1[k] = 0.0f;
    for (uint32_t k = threadIdx.x; k < 64 * 64; k += blockDim.x) T.gw2[k] = 0.0f;
    for (uint32_t k = threadIdx.x; k < 64; k += blockDim.x) T.gb1[k] = T.gb2[k] = T.gw3[k] = 0.0f;
    if (threadIdx.x == 0) T.gb3 = 0.0f;
    __syncthreads();
    const SmemMlp& S = T.S;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    __nv_bfloat16* xs = T.xs[warp];
    __nv_bfloat16* hs = T.hs[warp];
    __nv_bfloat16* ds = T.ds[warp];
    const float inv_b = 1.0f / (float)nrows;
    float loss_acc = 0.0f;
    for (uint32_t tile = blockIdx.x * 4 + warp; tile < (nrows + 15) / 16; tile += gridDim.x * 4) {
        float tgt = 0.0f;
        bool valid = false;
        if (lane < 16) {
            const uint32_t r = tile * 16 + lane;
            float f[9];
            valid = r < nrows;
            const uint32_t s = valid ? idx[r] : 0u;
            for (int k = 0; k < 9; ++k) f[k] = valid ? feat[(size_t)s * 9 + k] : 0.0f;
            store_row(S, f, xs + lane * 16);
            tgt = valid ? (target[s] - f[1] - S.tmean) / S.tstd : 0.0f;
        }
        __syncwarp();
        TileFwd F;
        tile_forward(S, xs, F);
        // dy per row (rows g and g+8), zero for padding rows
        const float t_lo = __shfl_sync(kAll, tgt, g), t_hi = __shfl_sync(kAll, tgt, g + 8);
        const bool v_lo = tile * 16 + g < nrows, v_hi = tile * 16 + g + 8 < nrows;
        const float e_lo = v_lo ? F.y_lo - t_lo : 0.0f, e_hi = v_hi ? F.y_hi - t_hi : 0.0f;
        if (t == 0) loss_acc += e_lo * e_lo + e_hi * e_hi;
        const float dy_lo = 2.0f * e_lo * inv_b, dy_hi = 2.0f * e_hi * inv_b;
        // layer 3 and dz2 (fp32), h1 / dz2 staged as bf16 for the tensor-core weight gradients
        float dz2[8][4];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int c = 8 * j + 2 * t;
            const float* z = F.z2[j];
            const float h00 = bf16r(silu(z[0])), h01 = bf16r(silu(z[1])), h10 = bf16r(silu(z[2])),
                        h11 = bf16r(silu(z[3]));
            float gw3a = dy_lo * h00 + dy_hi * h10, gw3b = dy_lo * h01 + dy_hi * h11;
            const float w3a = __bfloat162float(S.w3[c]), w3b = __bfloat162float(S.w3[c + 1]);
            dz2[j][0] = dy_lo * w3a * dsilu(z[0]);
            dz2[j][1] = dy_lo * w3b * dsilu(z[1]);
            dz2[j][2] = dy_hi * w3a * dsilu(z[2]);
            dz2[j][3] = dy_hi * w3b * dsilu(z[3]);
            float gb2a = dz2[j][0] + dz2[j][2], gb2b = dz2[j][1] + dz2[j][3];
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                gw3a += __shfl_xor_sync(kAll, gw3a, o);
                gw3b += __shfl_xor_sync(kAll, gw3b, o);
                gb2a += __shfl_xor_sync(kAll, gb2a, o);
                gb2b += __shfl_xor_sync(kAll, gb2b, o);
            }
            if (g == 0) {
                atomicAdd(&T.gw3[c], gw3a);
                atomicAdd(&T.gw3[c + 1], gw3b);
                atomicAdd(&T.gb2[c], gb2a);
                atomicAdd(&T.gb2[c + 1], gb2b);
            }
            const float* z1 = F.z1[j];
            hs[g * 64 + c] = __float2bfloat16_rn(silu(z1[0]));
            hs[g * 64 + c + 1] = __float2bfloat16_rn(silu(z1[1]));
            hs[(g + 8) * 64 + c] = __float2bfloat16_rn(silu(z1[2]));
            hs[(g + 8) * 64 + c + 1] = __float2bfloat16_rn(silu(z1[3]));
            ds[g * 64 + c] = __float2bfloat16_rn(dz2[j][0]);
            ds[g * 64 + c + 1] = __float2bfloat16_rn(dz2[j][1]);
            ds[(g + 8) * 64 + c] = __float2bfloat16_rn(dz2[j][2]);
            ds[(g + 8) * 64 + c + 1] = __float2bfloat16_rn(dz2[j][3]);
        }
        if (t == 0) atomicAdd(&T.gb3, dy_lo + dy_hi);
        __syncwarp();
        // dW2[out][in] = sum_rows dz2[row][out] * h1[row][in]   (M = out, N = in, K = 16 rows)
#pragma unroll 1
        for (int mt = 0; mt < 4; ++mt) {
            uint32_t a[4];
            const int mo = 16 * mt;
            a[0] = two(ds[(2 * t) * 64 + mo + g], ds[(2 * t + 1) * 64 + mo + g]);
            a[1] = two(ds[(2 * t) * 64 + mo + g + 8], ds[(2 * t + 1) * 64 + mo + g + 8]);
            a[2] = two(ds[(2 * t + 8) * 64 + mo + g], ds[(2 * t + 9) * 64 + mo + g]);
            a[3] = two(ds[(2 * t + 8) * 64 + mo + g + 8], ds[(2 * t + 9) * 64 + mo + g + 8]);
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const int ni = 8 * nt + g;
                mma16816(d, a, two(hs[(2 * t) * 64 + ni], hs[(2 * t + 1) * 64 + ni]),
                         two(hs[(2 * t + 8) * 64 + ni], hs[(2 * t + 9) * 64 + ni]));
                const int col = 8 * nt + 2 * t;
                atomicAdd(&T.gw2[(mo + g) * 64 + col], d[0]);
                atomicAdd(&T.gw2[(mo + g) * 64 + col + 1], d[1]);
                atomicAdd(&T.gw2[(mo + g + 8) * 64 + col], d[2]);
                atomicAdd(&T.gw2[(mo + g + 8) * 64 + col + 1], d[3]);
            }
        }
        // dh1 = dz2 x W2 (M = 16 rows, K = 64 out, N = 64 in); A from the dz2 registers, B[k=out][n=in] = W2[out][in]
        uint32_t ad[4][4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            ad[kk][0] = pack_bf16(dz2[2 * kk][0], dz2[2 * kk][1]);
            ad[kk][1] = pack_bf16(dz2[2 * kk][2], dz2[2 * kk][3]);
            ad[kk][2] = pack_bf16(dz2[2 * kk + 1][0], dz2[2 * kk + 1][1]);
            ad[kk][3] = pack_bf16(dz2[2 * kk + 1][2], dz2[2 * kk + 1][3]);
        }
        __syncwarp();
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float d[4] = {0.f, 0.f, 0.f, 0.f};
            const int ni = 8 * nt + g;
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const int ko = 16 * kk;
                mma16816(d, ad[kk], two(S.w2[(ko + 2 * t) * 64 + ni], S.w2[(ko + 2 * t + 1) * 64 + ni]),
                         two(S.w2[(ko + 2 * t + 8) * 64 + ni], S.w2[(ko + 2 * t + 9) * 64 + ni]));
            }
            // dz1 = dh1 * silu'(z1), staged (bf16) over dz2's buffer; db1
            const int c = 8 * nt + 2 * t;
            const float* z1 = F.z1[nt];
            const float q0 = d[0] * dsilu(z1[0]), q1 = d[1] * dsilu(z1[1]), q2 = d[2] * dsilu(z1[2]),
                        q3 = d[3] * dsilu(z1[3]);
            float gb1a = q0 + q2, gb1b = q1 + q3;
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                gb1a += __shfl_xor_sync(kAll, gb1a, o);
                gb1b += __shfl_xor_sync(kAll, gb1b, o);
            }
            if (g == 0) {
                atomicAdd(&T.gb1[c], gb1a);
                atomicAdd(&T.gb1[c + 1], gb1b);
            }
            __syncwarp();
            ds[g * 64 + c] = __float2bfloat16_rn(q0);
            ds[g * 64 + c + 1] = __float2bfloat16_rn(q1);
            ds[(g + 8) * 64 + c] = __float2bfloat16_rn(q2);
            ds[(g + 8) * 64 + c + 1] = __float2bfloat16_rn(q3);
        }
        __syncwarp();
        // dW1[out][in] = sum_rows dz1[row][out] * x[row][in]   (M = out, N = in (16), K = 16 rows)
#pragma unroll 1
        for (int mt = 0; mt < 4; ++mt) {
            uint32_t a[4];
            const int mo = 16 * mt;
            a[0] = two(ds[(2 * t) * 64 + mo + g], ds[(2 * t + 1) * 64 + mo + g]);
            a[1] = two(ds[(2 * t) * 64 + mo + g + 8], ds[(2 * t + 1) * 64 + mo + g + 8]);
            a[2] = two(ds[(2 * t + 8) * 64 + mo + g], ds[(2 * t + 9) * 64 + mo + g]);
            a[3] = two(ds[(2 * t + 8) * 64 + mo + g + 8], ds[(2 * t + 9) * 64 + mo + g + 8]);
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const int ni = 8 * nt + g;
                mma16816(d, a, two(xs[(2 * t) * 16 + ni], xs[(2 * t + 1) * 16 + ni]),
                         two(xs[(2 * t + 8) * 16 + ni], xs[(2 * t + 9) * 16 + ni]));
                const int col = 8 * nt + 2 * t;
                atomicAdd(&T.gw1[(mo + g) * 16 + col], d[0]);
                atomicAdd(&T.gw1[(mo + g) * 16 + col + 1], d[1]);
                atomicAdd(&T.gw1[(mo + g + 8) * 16 + col], d[2]);
                atomicAdd(&T.gw1[(mo + g + 8) * 16 + col + 1], d[3]);
            }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) loss_acc += __shfl_xor_sync(kAll, loss_acc, o);
    if (lane == 0) atomicAdd(loss, loss_acc);
    __syncthreads();
    // block partial gradients → global (fp32)
    for (uint32_t k = threadIdx.x; k < 64 * 9; k += blockDim.x) atomicAdd(&grads[k], T.gw1[(k / 9) * 16 + k % 9]);
    for (uint32_t k = threadIdx.x; k < 64; k += blockDim.x) {
        atomicAdd(&grads[576 + k], T.gb1[k]);
        atomicAdd(&grads[576 + 64 + 4096 + k], T.gb2[k]);
        atomicAdd(&grads[576 + 64 + 4096 + 64 + k], T.gw3[k]);
    }
    for (uint32_t k = threadIdx.x; k < 64 * 64; k += blockDim.x) atomicAdd(&grads[576 + 64 + k], T.gw2[k]);
    if (threadIdx.x == 0) atomicAdd(&grads[XPBD_MLP_PARAMS - 1], T.gb3);
}

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
                             uint32_t nrows, float* grads, float* loss, cudaStream_t st) {
    // the attribute is per device; setting it again is cheap and idempotent
    const size_t smem = sizeof(TrainSmem);
    if (cudaFuncSetAttribute(mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return cudaErrorInvalidValue;
    uint32_t grid = ((nrows + 15) / 16 + 3) / 4;
    if (grid > 296) grid = 296;
    if (grid == 0) grid = 1;
    mlp_train_kernel<<<grid, 128, smem, st>>>(mlp, feat, target, idx, nrows, grads, loss);
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
