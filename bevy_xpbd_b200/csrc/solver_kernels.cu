// XPBD substep kernels for sm_100a: predict/integrate, Jacobi and colored Gauss–Seidel distance-constraint solves,
// post-velocity, strain residual.
//
// Arithmetic follows the reference CPU solver src/xpbd_cpu.rs operation by operation with correctly rounded IEEE
// single-precision intrinsics (__fadd_rn/__fmul_rn/__fdiv_rn/__fsqrt_rn never contract into FMA), so the CUDA path
// reproduces the FP32 reference bit for bit:
//   predict_particle          xpbd_cpu.rs:38-65     (WGSL predict_copy_sim_to_jac, cloth_sim_jacobi.wgsl:85-121)
//   jacobi_edges_pass         xpbd_cpu.rs:139-184   (WGSL jacobi_edges :143-180)
//   jacobi_gather_particle    xpbd_cpu.rs:186-226   (WGSL jacobi_gather :182-218)
//   Gauss–Seidel sweep        xpbd_cpu.rs:344-386   (WGSL gs_edges, cloth_sim.wgsl:154-210)
//   post_velocity             xpbd_cpu.rs:393-409   (WGSL post_velocity :220-233)
//
// B200 design. One persistent kernel runs whole substeps: a grid-stride predict phase, then the inner iterations
// separated by a bounded grid barrier (no launch per iteration, no per-iteration λ clear launch). The Jacobi edge
// and gather passes are fused: each warp owns a tile of up to 32 consecutive particles; its lanes stride over the
// tile's incidences (coalesced 8-byte records), each lane computing one incidence's Δλ and correction, and the
// corrections are then summed per particle in the reference's neighbour order from shared memory — a deterministic
// warp-level segmented reduction without atomics. Finalize (velocity update) and the next substep's predict are
// fused into the last iteration, so a frame of S substeps × I iterations needs S·I grid barriers.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "xpbd_device.h"
#include "xpbd_fpdiv.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {

// ---------------------------------------------------------------------------------------------- grid barrier
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// atomicAdd with release semantics at GPU scope: the block's writes (ordered before it by __syncthreads) become
// visible to any thread that acquires the counter value it produces.
__device__ __forceinline__ unsigned atom_add_release(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.release.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// All blocks of the grid meet here. One atomic per block: block 0 adds 2^31 - (expected - 1), every other block adds
// 1, so the counter's top bit flips exactly when the last block arrives and the low bits return to their value;
// each block then polls for the flip. Each add is a release and the poll an acquire: the adds form one release
// sequence on the counter, so the load that sees the flip orders every block's earlier writes before the block's
// later reads (no separate fences). Waits are bounded: after `barrier_timeout_ns` (or once another block reported
// an error) the waiting block records XPBD_DEV_BARRIER_TIMEOUT and every caller returns false, so a launch that
// cannot complete (blocks not co-resident, forced test timeout) ends instead of hanging.
__device__ bool grid_barrier(const XpbdWorld& W, const XpbdDevParams& P) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        XpbdGridSync* gs = W.sync;
        const unsigned expected = gridDim.x + gs->expected_extra;
        const unsigned inc = (blockIdx.x == 0) ? (0x80000000u - (expected - 1u)) : 1u;
        const unsigned old = atom_add_release(&gs->count, inc);
        unsigned spins = 0;
        unsigned long long t0 = 0;
        while (((old ^ ld_acquire(&gs->count)) & 0x80000000u) == 0u) {
            ++spins;
            if ((spins & 255u) == 0u) {
                if (t0 == 0) t0 = global_ns();
                if (*(volatile int*)W.status != 0) { ok = 0; break; }
                if (global_ns() - t0 > P.barrier_timeout_ns || spins > (1u << 30)) {
                    set_status(W.status, XPBD_DEV_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                if (spins > (1u << 16)) __nanosleep(128);
            }
        }
        s_ok = ok;  // the acquiring load that saw the flip orders the other blocks' writes before what follows
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ bool status_clear(const XpbdWorld& W) { return *(volatile int*)W.status == 0; }

// ---------------------------------------------------------------------------------------------- predict phase
// Grid-stride over particles. Optionally finalizes a pending substep (positions in jac[pend]) first, then predicts
// into jac[start]. Pinned particles are written to both ping-pong buffers (they never move).
// `range_flag` (optional): set to 1 when a predicted or pinned position has a coordinate outside the range of the
// unchecked shared-reciprocal division (coord_outside_fast_range).
__device__ void predict_phase(const XpbdWorld& W, const XpbdDevParams& P, bool finalize_pending, uint32_t pend,
                              uint32_t start, bool predict, unsigned* range_flag = nullptr) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n; i += stride) {
        float4 xo4 = W.x[i];
        F3 xo = f3(xo4);
        const float w = xo4.w;
        if (w <= 0.0f) {
            if (predict) {
                W.jac[0][i] = xo4;
                W.jac[1][i] = xo4;
                if (range_flag && (coord_outside_fast_range(xo4.x) | coord_outside_fast_range(xo4.y) |
                                   coord_outside_fast_range(xo4.z)))
                    *range_flag = 1u;
            }
            continue;
        }
        float4 vo4 = W.v[i];
        F3 vel = f3(vo4);
        if (finalize_pending) {
            F3 xn = finalize_particle(f3(W.jac[pend][i]), xo, vel, P, W.status);
            W.x[i] = make_float4(xn.x, xn.y, xn.z, w);
            W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
            xo = xn;
        }
        if (predict) {
            F3 pos = predict_w(W, i, xo, vel, P);
            W.jac[start][i] = make_float4(pos.x, pos.y, pos.z, w);
            if (range_flag && (coord_outside_fast_range(pos.x) | coord_outside_fast_range(pos.y) |
                               coord_outside_fast_range(pos.z)))
                *range_flag = 1u;
        }
    }
}

// ---------------------------------------------------------------------------------------------- Jacobi tile
enum TailMode : uint32_t { kTailNone = 0, kTailFinalize = 1, kTailFinalizePredict = 2 };

constexpr uint32_t kTileChunk = 512;  // incidences staged per warp pass (a 32-particle cloth tile holds ~384)

// One Jacobi iteration for one warp tile (jacobi_edges + jacobi_gather fused). Phase A: the lanes stride over the
// tile's incidences (coalesced 8-byte records), each computing one incidence's correction — the reference's Δλ of
// its constraint (recomputed identically from either endpoint) times n̂·w_self — into shared memory. Phase B: each
// particle's lane sums its own incidences from shared memory in neighbour-table order (the reference's order), so
// the result is bit-identical to jacobi_gather_particle. `sc` is the warp's 3 x kTileChunk staging area.
__device__ __forceinline__ void jacobi_tile(const XpbdWorld& W, const XpbdDevParams& P, uint32_t tile,
                                            const float4* __restrict__ jin, float4* __restrict__ jout, float* sc,
                                            uint32_t lane, TailMode tail) {
    const XpbdTile t = W.tiles[tile];
    const uint32_t cnt = t.count;
    const bool has_row = lane < cnt;
    const uint32_t r = t.first + lane;
    uint32_t rs = 0, re = 0;
    float4 ps = make_float4(0.f, 0.f, 0.f, 0.f);
    if (has_row) {
        rs = W.row_off[r];
        re = W.row_off[r + 1];
        ps = jin[r];
    }
    const uint32_t I0 = __shfl_sync(kFull, rs, 0);
    const uint32_t I1 = __shfl_sync(kFull, re, cnt - 1);
    const float* pal = W.palette_comp + (uint32_t)t.cloth * XPBD_PALETTE;
    const bool persist = P.lambda_mode != 0u;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    for (uint32_t cb = I0; cb < I1; cb += kTileChunk) {
        const uint32_t ce = min(I1, cb + kTileChunk);
        for (uint32_t k = cb + lane; k < ce + ((32u - ((ce - cb) & 31u)) & 31u); k += 32) {
            // owner row of incidence k: smallest rr with row_end[rr] > k (binary search over the lanes' row ends)
            uint32_t lo = 0, hi = cnt;
#pragma unroll
            for (int it = 0; it < 6; ++it) {
                const uint32_t mid = (lo + hi) >> 1;
                const uint32_t em = __shfl_sync(kFull, re, mid & 31u);
                if (lo < hi) {
                    if (em > k) hi = mid; else lo = mid + 1;
                }
            }
            const uint32_t rr = lo & 31u;
            const float sx = __shfl_sync(kFull, ps.x, rr);
            const float sy = __shfl_sync(kFull, ps.y, rr);
            const float sz = __shfl_sync(kFull, ps.z, rr);
            const float sw = __shfl_sync(kFull, ps.w, rr);
            if (k >= ce) continue;
            F3 c = {0.0f, 0.0f, 0.0f};
            const uint2 rec = W.inc[k];
            const uint32_t other = rec.x & XPBD_OTHER_MASK;
            if (other >= W.n) {  // corrupt table: record and skip
                set_status(W.status, XPBD_DEV_INDEX);
                continue;
            }
            const float rest = __uint_as_float(rec.y);
            const float4 po = jin[other];
            const F3 gv = sub3(F3{sx, sy, sz}, f3(po));
            const float len = len3(gv);
            float lam_next = 0.0f;
            bool write_lam = persist;
            if (!(len < 1e-8f)) {
                const F3 nrm = div3(gv, len);
                const float C = __fsub_rn(len, rest);
                const float alpha_t = __fmul_rn(inc_compliance(W, pal, rec, k), P.inv_dt_sq);
                const float wsum = __fadd_rn(__fadd_rn(sw, po.w), alpha_t);
                float dlam = 0.0f;
                if (!(wsum < 1e-8f)) {
                    const float lam = persist ? W.inc_lambda[k] : 0.0f;
                    dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, lam)), wsum);
                    lam_next = __fadd_rn(lam, dlam);
                } else {
                    write_lam = persist && tail == kTailFinalizePredict;
                }
                c = mul3(mul3(nrm, sw), dlam);
            } else {
                write_lam = persist && tail == kTailFinalizePredict;
            }
            if (write_lam) W.inc_lambda[k] = (tail == kTailFinalizePredict) ? 0.0f : lam_next;
            const uint32_t s = k - cb;
            sc[s] = c.x;
            sc[kTileChunk + s] = c.y;
            sc[2 * kTileChunk + s] = c.z;
        }
        __syncwarp();
        if (has_row && re > cb && rs < ce) {
            const uint32_t a = (rs > cb ? rs : cb) - cb;
            const uint32_t b = (re < ce ? re : ce) - cb;
#pragma unroll 4
            for (uint32_t q = a; q < b; ++q) {
                ax = __fadd_rn(ax, sc[q]);
                ay = __fadd_rn(ay, sc[kTileChunk + q]);
                az = __fadd_rn(az, sc[2 * kTileChunk + q]);
            }
        }
        __syncwarp();
    }
    if (!has_row || ps.w <= 0.0f) return;  // pinned: both buffers already hold the fixed position
    F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
    if (P.relaxation == 1u && re > rs) delta = div3(delta, (float)(re - rs));
    delta = clamp_correction(delta);
    F3 xn = add3(f3(ps), delta);
    if (tail == kTailNone) {
        jout[r] = make_float4(xn.x, xn.y, xn.z, ps.w);
        return;
    }
    // fused post_velocity (+ next substep's predict)
    const F3 xo = f3(W.x[r]);
    F3 vel = f3(W.v[r]);
    xn = finalize_particle(xn, xo, vel, P, W.status);
    W.x[r] = make_float4(xn.x, xn.y, xn.z, ps.w);
    W.v[r] = make_float4(vel.x, vel.y, vel.z, 0.0f);
    if (tail == kTailFinalizePredict) {
        F3 pos = predict_w(W, r, xn, vel, P);
        jout[r] = make_float4(pos.x, pos.y, pos.z, ps.w);
    } else {
        jout[r] = make_float4(xn.x, xn.y, xn.z, ps.w);
    }
}

// Persistent Jacobi kernel: `substeps` substeps of the whole batch.
//   flags & kBeginFinalize : a previous substep's result waits in jac[pend] (e.g. after collision) — finalize it
//   flags & kEndFinalize   : finalize the last substep in place; otherwise its result stays in jac[final]
// The predict of the first substep writes jac[start]; iteration k of a substep reads buffer (b+k)&1.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) jacobi_persistent_kernel(XpbdWorld W, uint32_t flags, uint32_t substeps,
                                                                  uint32_t pend, uint32_t start) {
    extern __shared__ float s_contrib[];  // (BLOCK/32) x 3 x kTileChunk floats
    if (!status_clear(W)) return;
    const XpbdDevParams P = *W.params;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t gwarp = blockIdx.x * (BLOCK / 32) + warp;
    const uint32_t nwarps = gridDim.x * (BLOCK / 32);
    float* sc = s_contrib + warp * 3 * kTileChunk;
    const bool persist = P.lambda_mode != 0u;

    predict_phase(W, P, (flags & kBeginFinalize) != 0u, pend, start, true);
    if (persist) {
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < W.n_inc; k += stride) W.inc_lambda[k] = 0.0f;
    }
    if (!grid_barrier(W, P)) return;
    uint32_t b = start;
    const uint32_t I = P.iterations;
    for (uint32_t s = 0; s < substeps; ++s) {
        const bool last_sub = (s + 1 == substeps);
        if (I == 0) {  // no constraint iterations: the predicted positions are the result (xpbd_cpu.rs:302-309)
            // finalize / re-predict per particle without reading neighbours
            const uint32_t stride = gridDim.x * blockDim.x;
            const bool fin = !last_sub || (flags & kEndFinalize);
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n && fin; i += stride) {
                float4 p4 = W.jac[b][i];
                if (p4.w <= 0.0f) continue;
                const F3 xo = f3(W.x[i]);
                F3 vel = f3(W.v[i]);
                F3 xn = finalize_particle(f3(p4), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                if (!last_sub) {
                    F3 pos = predict_w(W, i, xn, vel, P);
                    W.jac[b][i] = make_float4(pos.x, pos.y, pos.z, p4.w);
                }
            }
            if (!last_sub && !grid_barrier(W, P)) return;
            continue;
        }
        for (uint32_t k = 0; k < I; ++k) {
            const float4* jin = W.jac[(b + k) & 1u];
            float4* jout = W.jac[(b + k + 1) & 1u];
            TailMode tail = kTailNone;
            if (k + 1 == I) {
                if (!last_sub) tail = kTailFinalizePredict;
                else if (flags & kEndFinalize) tail = kTailFinalize;
            }
            for (uint32_t tile = gwarp; tile < W.n_tiles; tile += nwarps) jacobi_tile(W, P, tile, jin, jout, sc, lane, tail);
            const bool very_last = last_sub && (k + 1 == I);
            if (!very_last && !grid_barrier(W, P)) return;
        }
        b = (b + I) & 1u;
    }
}

// ---------------------------------------------------------------------------------------------- Jacobi rows
// Thread per particle over the neighbour table (no shared memory, full occupancy). Each incidence recomputes its
// constraint's Δλ exactly as jacobi_edges would (identical from either endpoint); the contributions of four
// consecutive incidences are evaluated as independent dependency chains and then added in neighbour-table order,
// so the sum is the reference's sequential one.
// One incidence of row i (reference jacobi_edges recomputed from this endpoint, then its jacobi_gather term): the
// correction (n̂·w_i)·Δλ, or zero where the reference skips the constraint (|d| < 1e-8) or has Δλ = 0 (w sum < 1e-8).
// Branch-free: a skipped term is selected as +0, which leaves the running sum unchanged (the sum starts at +0 and
// adding terms never yields -0).
// UNCHECKED: n̂ by fpdiv3_unchecked — only when the pass's coordinate check found every position in range.
// PLAIN: XpbdDevParams::plain_terms holds — α̃ is finite (so −C − α̃·0 = −C) and the w sum of a free row's
// constraint is >= its own inverse mass >= 1e-8 (so only the length test can skip the term).
template <bool UNCHECKED, bool PLAIN>
__device__ __forceinline__ F3 row_term(const F3 self, float wi, const float4 po, float rest, float alpha_t) {
    const F3 gv = sub3(self, f3(po));
    const float len = len3(gv);
    F3 nrm;
    if (UNCHECKED) {
        fpdiv3_unchecked(gv.x, gv.y, gv.z, len, nrm.x, nrm.y, nrm.z);  // a skipped term (len < 1e-8) is discarded
    } else {
        nrm = div3(gv, len);
    }
    const float C = __fsub_rn(len, rest);
    const float wsum = __fadd_rn(__fadd_rn(wi, po.w), alpha_t);
    const float dlam = __fdiv_rn(PLAIN ? -C : __fsub_rn(-C, __fmul_rn(alpha_t, 0.0f)), wsum);
    const bool use = PLAIN ? !(len < 1e-8f) : !(len < 1e-8f) && !(wsum < 1e-8f);
    return {use ? __fmul_rn(__fmul_rn(nrm.x, wi), dlam) : 0.0f, use ? __fmul_rn(__fmul_rn(nrm.y, wi), dlam) : 0.0f,
            use ? __fmul_rn(__fmul_rn(nrm.z, wi), dlam) : 0.0f};
}

// unchecked: every position of this pass's input is in the fast-division range; range_next: the flag of the next
// pass, set when a position this call writes is not.
__device__ __forceinline__ void jacobi_row(const XpbdWorld& W, const XpbdDevParams& P, uint32_t i,
                                           const float4* __restrict__ jin, float4* __restrict__ jout,
                                           TailMode tail, bool unchecked, unsigned* range_next) {
    const float4 ps = jin[i];
    if (ps.w <= 0.0f) {  // pinned: not moved, but its position is read by its neighbours in the next pass too
        if (coord_outside_fast_range(ps.x) | coord_outside_fast_range(ps.y) | coord_outside_fast_range(ps.z))
            *range_next = 1u;
        return;
    }
    const uint32_t rs = W.row_off[i], re = W.row_off[i + 1];
    const bool persist = P.lambda_mode != 0u;
    const float* __restrict__ pal = W.palette_comp + (uint32_t)W.row_cloth[i] * XPBD_PALETTE;
    const uint2* __restrict__ recs = W.inc;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    const F3 self = f3(ps);
    if (!persist) {
        // λ = 0 at every pass (reference mode): pairs of independent terms, then the remainder, summed in
        // incidence order. The compliance source (palette or per-incidence array) is fixed per launch.
        auto sum_terms = [&](auto unchecked_tag, auto plain_tag, auto wide_tag) {
            constexpr bool U = decltype(unchecked_tag)::value, PL = decltype(plain_tag)::value;
            constexpr bool WIDE = decltype(wide_tag)::value;
            auto comp_of = [&](uint2 rec, uint32_t k) { return WIDE ? W.inc_comp[k] : pal[rec.x >> 28]; };
            uint32_t k = rs;
            for (; k + 2 <= re; k += 2) {  // pairs: measured faster than groups of four or six
                F3 c[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const uint2 rec = recs[k + u];
                    c[u] = row_term<U, PL>(self, ps.w, jin[rec.x & XPBD_OTHER_MASK], __uint_as_float(rec.y),
                                           __fmul_rn(comp_of(rec, k + u), P.inv_dt_sq));
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    ax = __fadd_rn(ax, c[u].x);
                    ay = __fadd_rn(ay, c[u].y);
                    az = __fadd_rn(az, c[u].z);
                }
            }
            for (; k < re; ++k) {
                const uint2 rec = recs[k];
                const F3 c = row_term<U, PL>(self, ps.w, jin[rec.x & XPBD_OTHER_MASK], __uint_as_float(rec.y),
                                             __fmul_rn(comp_of(rec, k), P.inv_dt_sq));
                ax = __fadd_rn(ax, c.x);
                ay = __fadd_rn(ay, c.y);
                az = __fadd_rn(az, c.z);
            }
        };
        const std::true_type yes;
        const std::false_type no;
        if (W.inc_comp) {  // batches with wide compliance sets
            if (unchecked)
                sum_terms(yes, no, yes);
            else
                sum_terms(no, no, yes);
        } else if (unchecked && P.plain_terms)
            sum_terms(yes, yes, no);
        else if (unchecked)
            sum_terms(yes, no, no);
        else
            sum_terms(no, no, no);
    } else {
        for (uint32_t k = rs; k < re; k += 4) {
            float cx[4], cy[4], cz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                cx[u] = cy[u] = cz[u] = 0.0f;
                const uint32_t kk = k + u;
                if (kk >= re) continue;
                const uint2 rec = recs[kk];
                const float4 po = jin[rec.x & XPBD_OTHER_MASK];
                const F3 gv = sub3(self, f3(po));
                const float len = len3(gv);
                if (len < 1e-8f) {
                    if (tail == kTailFinalizePredict) W.inc_lambda[kk] = 0.0f;
                    continue;
                }
                const F3 nrm = div3(gv, len);
                const float C = __fsub_rn(len, __uint_as_float(rec.y));
                const float alpha_t = __fmul_rn(inc_compliance(W, pal, rec, kk), P.inv_dt_sq);
                const float wsum = __fadd_rn(__fadd_rn(ps.w, po.w), alpha_t);
                float dlam = 0.0f;
                if (!(wsum < 1e-8f)) {
                    const float lam = W.inc_lambda[kk];
                    dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, lam)), wsum);
                    W.inc_lambda[kk] = (tail == kTailFinalizePredict) ? 0.0f : __fadd_rn(lam, dlam);
                } else if (tail == kTailFinalizePredict) {
                    W.inc_lambda[kk] = 0.0f;
                }
                cx[u] = __fmul_rn(__fmul_rn(nrm.x, ps.w), dlam);
                cy[u] = __fmul_rn(__fmul_rn(nrm.y, ps.w), dlam);
                cz[u] = __fmul_rn(__fmul_rn(nrm.z, ps.w), dlam);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k + u < re) {
                    ax = __fadd_rn(ax, cx[u]);
                    ay = __fadd_rn(ay, cy[u]);
                    az = __fadd_rn(az, cz[u]);
                }
        }
    }
    F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
    if (P.relaxation == 1u && re > rs) delta = div3(delta, (float)(re - rs));
    delta = clamp_correction(delta);
    F3 xn = add3(self, delta);
    auto note_range = [&](const F3& q) {
        if (coord_outside_fast_range(q.x) | coord_outside_fast_range(q.y) | coord_outside_fast_range(q.z))
            *range_next = 1u;
    };
    if (tail == kTailNone) {
        jout[i] = make_float4(xn.x, xn.y, xn.z, ps.w);
        note_range(xn);
        return;
    }
    const F3 xo = f3(W.x[i]);
    F3 vel = f3(W.v[i]);
    xn = finalize_particle(xn, xo, vel, P, W.status);
    W.x[i] = make_float4(xn.x, xn.y, xn.z, ps.w);
    W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
    if (tail == kTailFinalizePredict) {
        const F3 pos = predict_w(W, i, xn, vel, P);
        jout[i] = make_float4(pos.x, pos.y, pos.z, ps.w);
        note_range(pos);
    } else {
        jout[i] = make_float4(xn.x, xn.y, xn.z, ps.w);
        note_range(xn);
    }
}

template <int BLOCK>
__device__ __forceinline__ void jacobi_rows_body(const XpbdWorld& W, uint32_t flags, uint32_t substeps, uint32_t pend,
                                                 uint32_t start) {
    if (!status_clear(W)) return;
    const XpbdDevParams P = *W.params;
    const bool persist = P.lambda_mode != 0u;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    // Pass p of this launch reads range slot p % 3 (written while its input positions were written: by the predict
    // phase for p = 0, by pass p - 1 otherwise) and clears slot (p + 2) % 3, last read by pass p - 1. Slots only ever
    // get set between clears, so a stale value can only force the exact division, never skip it.
    predict_phase(W, P, (flags & kBeginFinalize) != 0u, pend, start, true, W.div_exact);
    if (persist)
        for (uint32_t k = gtid; k < W.n_inc; k += gstride) W.inc_lambda[k] = 0.0f;
    if (!grid_barrier(W, P)) return;
    uint32_t b = start, pass = 0;
    const uint32_t I = P.iterations;
    for (uint32_t s = 0; s < substeps; ++s) {
        const bool last_sub = (s + 1 == substeps);
        if (I == 0) {
            const bool fin = !last_sub || (flags & kEndFinalize);
            for (uint32_t i = gtid; i < W.n && fin; i += gstride) {
                float4 p4 = W.jac[b][i];
                if (p4.w <= 0.0f) continue;
                const F3 xo = f3(W.x[i]);
                F3 vel = f3(W.v[i]);
                F3 xn = finalize_particle(f3(p4), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                if (!last_sub) {
                    F3 pos = predict_w(W, i, xn, vel, P);
                    W.jac[b][i] = make_float4(pos.x, pos.y, pos.z, p4.w);
                }
            }
            if (!last_sub && !grid_barrier(W, P)) return;
            continue;
        }
        for (uint32_t k = 0; k < I; ++k) {
            const float4* jin = W.jac[(b + k) & 1u];
            float4* jout = W.jac[(b + k + 1) & 1u];
            TailMode tail = kTailNone;
            if (k + 1 == I) {
                if (!last_sub) tail = kTailFinalizePredict;
                else if (flags & kEndFinalize) tail = kTailFinalize;
            }
            const bool unchecked = *(volatile unsigned*)&W.div_exact[pass % 3u] == 0u;
            if (gtid == 0) W.div_exact[(pass + 2u) % 3u] = 0u;
            unsigned* range_next = W.div_exact + (pass + 1u) % 3u;
            for (uint32_t i = gtid; i < W.n; i += gstride)
                jacobi_row(W, P, i, jin, jout, tail, unchecked, range_next);
            ++pass;
            const bool very_last = last_sub && (k + 1 == I);
            if (!very_last && !grid_barrier(W, P)) return;
        }
        b = (b + I) & 1u;
    }
}

// Thread per particle over the row-ordered incidence table (kernel id 5).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) jacobi_row_kernel(XpbdWorld W, uint32_t flags, uint32_t substeps,
                                                           uint32_t pend, uint32_t start) {
    jacobi_rows_body<BLOCK>(W, flags, substeps, pend, start);
}

// ---------------------------------------------------------------------------------------------- convergence solve
// Jacobi substep with λ kept over the substep, iterated until the pre-update residual max |C + α̃λ|/rest <= tolerance
// (at most max_iterations passes), optionally warm-started from λ0: positions move by the reference gather with Δλ
// replaced by λ0 and λ starts at λ0, unless that leaves a cloth's residual above its plain (λ = 0) start — then the
// cloth falls back to the plain start for this substep. Thread per particle (row), fixed particle→thread mapping
// across phases, so a particle's own incidences (and their λ copies) are only touched by its thread.
__device__ __forceinline__ float residual_of(float len, float rest, float alpha_t, float lam) {
    return __fdiv_rn(fabsf(__fadd_rn(__fsub_rn(len, rest), __fmul_rn(alpha_t, lam))), rest);
}

__device__ __forceinline__ void block_max_atomic(float v, unsigned* dst) {
    __shared__ float s_max[32];
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s_max[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (blockDim.x >> 5) ? s_max[lane] : 0.0f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
        if (lane == 0 && v > 0.0f) atomicMax(dst, __float_as_uint(v));
    }
}

// Predict into jac[0] (pinned: both buffers) and clear the per-substep residual slots.
__global__ void converge_predict_kernel(XpbdWorld W) {
    const XpbdDevParams P = *W.params;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    for (uint32_t k = gtid; k < 2 * W.n_cloths; k += gstride) W.cloth_res[k] = 0u;
    for (uint32_t k = gtid; k < 3 * W.n_cloths; k += gstride) W.cloth_ires[k] = 0u;
    for (uint32_t k = gtid; k < W.n_cloths; k += gstride) W.cloth_iters[k] = 0u;
    for (uint32_t k = gtid; k < XPBD_MAX_CONVERGE_ITERS; k += gstride) W.iter_res[k] = 0u;
    for (uint32_t i = gtid; i < W.n; i += gstride) {
        const float4 x4 = W.x[i];
        if (x4.w <= 0.0f) {
            W.jac[0][i] = x4;
            W.jac[1][i] = x4;
            continue;
        }
        F3 vel = f3(W.v[i]);
        const F3 pos = predict_w(W, i, f3(x4), vel, P);
        W.jac[0][i] = make_float4(pos.x, pos.y, pos.z, x4.w);
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) jacobi_converge_kernel(XpbdWorld W, uint32_t warm) {
    if (!status_clear(W)) return;
    const XpbdDevParams P = *W.params;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    const float* lam0 = W.warm_lam_inc;
    if (warm) {
        // plain start residual (λ = 0) per cloth, and the warm-started positions into jac[1]
        for (uint32_t i = gtid; i < W.n; i += gstride) {
            const float4 ps = W.jac[0][i];
            if (ps.w <= 0.0f) continue;
            const uint32_t rs = W.row_off[i], re = W.row_off[i + 1];
            const float* pal = W.palette_comp + (uint32_t)W.row_cloth[i] * XPBD_PALETTE;
            float rmax = 0.0f, ax = 0.0f, ay = 0.0f, az = 0.0f;
            for (uint32_t k = rs; k < re; ++k) {
                const uint2 rec = W.inc[k];
                const float4 po = W.jac[0][rec.x & XPBD_OTHER_MASK];
                const F3 gv = sub3(f3(ps), f3(po));
                const float len = len3(gv);
                const float alpha_t = __fmul_rn(inc_compliance(W, pal, rec, k), P.inv_dt_sq);
                rmax = fmaxf(rmax, residual_of(len, __uint_as_float(rec.y), alpha_t, 0.0f));
                if (len < 1e-8f) continue;
                const F3 nrm = div3(gv, len);
                const float l0 = lam0[k];
                ax = __fadd_rn(ax, __fmul_rn(__fmul_rn(nrm.x, ps.w), l0));
                ay = __fadd_rn(ay, __fmul_rn(__fmul_rn(nrm.y, ps.w), l0));
                az = __fadd_rn(az, __fmul_rn(__fmul_rn(nrm.z, ps.w), l0));
            }
            if (rmax > 0.0f) atomicMax(&W.cloth_res[2 * W.row_cloth[i]], __float_as_uint(rmax));
            F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
            if (P.relaxation == 1u && re > rs) delta = div3(delta, (float)(re - rs));
            delta = clamp_correction(delta);
            const F3 xn = add3(f3(ps), delta);
            W.jac[1][i] = make_float4(xn.x, xn.y, xn.z, ps.w);
        }
        if (!grid_barrier(W, P)) return;
        // warm start residual per cloth (positions jac[1], λ = λ0)
        for (uint32_t i = gtid; i < W.n; i += gstride) {
            const float4 ps = W.jac[1][i];
            if (ps.w <= 0.0f) continue;
            const uint32_t rs = W.row_off[i], re = W.row_off[i + 1];
            const float* pal = W.palette_comp + (uint32_t)W.row_cloth[i] * XPBD_PALETTE;
            float rmax = 0.0f;
            for (uint32_t k = rs; k < re; ++k) {
                const uint2 rec = W.inc[k];
                const float len = len3(sub3(f3(ps), f3(W.jac[1][rec.x & XPBD_OTHER_MASK])));
                const float alpha_t = __fmul_rn(inc_compliance(W, pal, rec, k), P.inv_dt_sq);
                rmax = fmaxf(rmax, residual_of(len, __uint_as_float(rec.y), alpha_t, lam0[k]));
            }
            if (rmax > 0.0f) atomicMax(&W.cloth_res[2 * W.row_cloth[i] + 1], __float_as_uint(rmax));
        }
        if (!grid_barrier(W, P)) return;
        // keep the warm start where it does not raise the cloth's residual
        for (uint32_t c = gtid; c < W.n_cloths; c += gstride)
            if (__uint_as_float(W.cloth_res[2 * c + 1]) > __uint_as_float(W.cloth_res[2 * c]))
                atomicAdd(&W.cstats->fallbacks, 1ull);
        for (uint32_t i = gtid; i < W.n; i += gstride) {
            const uint32_t c = W.row_cloth[i];
            const bool keep = !(__uint_as_float(W.cloth_res[2 * c + 1]) > __uint_as_float(W.cloth_res[2 * c]));
            if (keep) W.jac[0][i] = W.jac[1][i];
            const uint32_t rs = W.row_off[i], re = W.row_off[i + 1];
            for (uint32_t k = rs; k < re; ++k) W.inc_lambda[k] = keep ? lam0[k] : 0.0f;
        }
    } else {
        for (uint32_t k = gtid; k < W.n_inc; k += gstride) W.inc_lambda[k] = 0.0f;
    }
    if (!grid_barrier(W, P)) return;
    // Iterations, per cloth: residual of the state before each update pass, checked after the pass; a cloth whose
    // residual was at or below the tolerance stops (its iterate is carried over unchanged) and the loop ends when no
    // cloth is left — each cloth takes the passes it would take alone. Per-cloth residuals rotate over three slots:
    // slot it%3 is written in iteration it, read after its barrier, and cleared in iteration it+2.
    uint32_t cur = 0, it = 0;
    const uint32_t maxit = min(P.max_iterations, (uint32_t)XPBD_MAX_CONVERGE_ITERS);
    const uint32_t nc = W.n_cloths, lane = threadIdx.x & 31u;
    while (it < maxit) {
        const float4* jin = W.jac[cur];
        float4* jout = W.jac[cur ^ 1u];
        const unsigned* prev_res = W.cloth_ires + ((it + 2u) % 3u) * nc;
        unsigned* cur_res = W.cloth_ires + (it % 3u) * nc;
        float rmax = 0.0f;
        for (uint32_t base = gtid - lane; base < W.n; base += gstride) {  // warp-uniform trip count
            const uint32_t i = base + lane;
            float ri = 0.0f;
            uint32_t ci = 0u;
            if (i < W.n) {
                const float4 ps = jin[i];
                ci = W.row_cloth[i];
                const bool active = it == 0u || __uint_as_float(prev_res[ci]) > P.tolerance;
                if (!active) {
                    jout[i] = ps;
                } else if (ps.w > 0.0f) {
                    const uint32_t rs = W.row_off[i], re = W.row_off[i + 1];
                    const float* pal = W.palette_comp + ci * XPBD_PALETTE;
                    float ax = 0.0f, ay = 0.0f, az = 0.0f;
                    for (uint32_t k = rs; k < re; ++k) {
                        const uint2 rec = W.inc[k];
                        const float4 po = jin[rec.x & XPBD_OTHER_MASK];
                        const F3 gv = sub3(f3(ps), f3(po));
                        const float len = len3(gv);
                        const float rest = __uint_as_float(rec.y);
                        const float alpha_t = __fmul_rn(inc_compliance(W, pal, rec, k), P.inv_dt_sq);
                        const float lam = W.inc_lambda[k];
                        ri = fmaxf(ri, residual_of(len, rest, alpha_t, lam));
                        if (len < 1e-8f) continue;
                        const F3 nrm = div3(gv, len);
                        const float C = __fsub_rn(len, rest);
                        const float wsum = __fadd_rn(__fadd_rn(ps.w, po.w), alpha_t);
                        if (wsum < 1e-8f) continue;
                        const float dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, lam)), wsum);
                        W.inc_lambda[k] = __fadd_rn(lam, dlam);
                        ax = __fadd_rn(ax, __fmul_rn(__fmul_rn(nrm.x, ps.w), dlam));
                        ay = __fadd_rn(ay, __fmul_rn(__fmul_rn(nrm.y, ps.w), dlam));
                        az = __fadd_rn(az, __fmul_rn(__fmul_rn(nrm.z, ps.w), dlam));
                    }
                    F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
                    if (P.relaxation == 1u && re > rs) delta = div3(delta, (float)(re - rs));
                    delta = clamp_correction(delta);
                    const F3 xn = add3(f3(ps), delta);
                    jout[i] = make_float4(xn.x, xn.y, xn.z, ps.w);
                }
            }
            // per-cloth max: one atomic per cloth present in the warp
            const bool has = ri > 0.0f;
            const unsigned hm = __ballot_sync(kFull, has);
            if (has) {
                const unsigned grp = __match_any_sync(hm, ci);
                const unsigned m = __reduce_max_sync(grp, __float_as_uint(ri));
                if (lane == (uint32_t)(__ffs(grp) - 1)) atomicMax(&cur_res[ci], m);
            }
            rmax = fmaxf(rmax, ri);
        }
        for (uint32_t c = gtid; c < nc; c += gstride) {
            W.cloth_ires[((it + 1u) % 3u) * nc + c] = 0u;
            if (it == 0u || __uint_as_float(prev_res[c]) > P.tolerance) W.cloth_iters[c] += 1u;
        }
        block_max_atomic(rmax, &W.iter_res[it]);
        if (!grid_barrier(W, P)) return;
        const float res = __uint_as_float(*(volatile unsigned*)&W.iter_res[it]);
        cur ^= 1u;
        ++it;
        if (res <= P.tolerance) break;
    }
    for (uint32_t c = gtid; c < nc; c += gstride) {
        atomicAdd(&W.cstats->iterations, (unsigned long long)W.cloth_iters[c]);
        atomicMax(&W.cstats->max_iterations, W.cloth_iters[c]);
    }
    if (gtid == 0) {
        atomicAdd(&W.cstats->substeps, (unsigned long long)nc);
        W.cstats->last_iterations = it;
    }
    // finalize (post_velocity) from the final iterate; pinned particles keep x, v
    for (uint32_t i = gtid; i < W.n; i += gstride) {
        const float4 p4 = W.jac[cur][i];
        if (p4.w <= 0.0f) continue;
        const F3 xo = f3(W.x[i]);
        F3 vel = f3(W.v[i]);
        const F3 xn = finalize_particle(f3(p4), xo, vel, P, W.status);
        W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
        W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
    }
}

// ---------------------------------------------------------------------------------------------- Jacobi patches
// Each CTA walks its patches (pid = blockIdx.x + m*gridDim.x). Per patch: (1) the patch's table blob was fetched into
// shared memory by one TMA bulk copy issued one patch ahead (cp.async.bulk, completion on an mbarrier, L2 evict-first
// so the streamed tables do not push the particle buffers out of L2); (2) its particles + halo were gathered into
// shared memory with cp.async while the previous patch was finishing; (3) every constraint is solved once
// (reference jacobi_edges: Δλ and n̂ = (p_i - p_j)/len) into shared memory; (4) each owned particle sums its
// incidences in neighbour-table order (reference jacobi_gather: (±n̂·w)·Δλ) — bit-identical to the reference, with
// each constraint's square root and divisions evaluated once instead of once per endpoint.
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void bulk_g2s_evict_first(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "{\n\t.reg .b64 pol;\n\tcreatepolicy.fractional.L2::evict_first.b64 pol, 1.0;\n\t"
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], pol;"
        "\n\t}" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Bounded wait on phase `parity`; false when the limit was reached.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ uint32_t align16(uint32_t b) { return (b + 15u) & ~15u; }

struct PatchView {
    const uint32_t* parts;
    const uint2* con;
    const uint32_t* gofs;
    const uint16_t* slots;
};
__device__ __forceinline__ PatchView patch_view(const unsigned char* blob, const XpbdPatch& pt) {
    PatchView v;
    const uint32_t nl = (uint32_t)pt.np + pt.nh;
    v.parts = reinterpret_cast<const uint32_t*>(blob);
    const unsigned char* c = blob + align16(4u * nl);
    v.con = reinterpret_cast<const uint2*>(c);
    const unsigned char* g = c + align16(8u * pt.nc);
    v.gofs = reinterpret_cast<const uint32_t*>(g);
    v.slots = reinterpret_cast<const uint16_t*>(g + align16(4u * ((uint32_t)pt.np + 1u)));
    return v;
}

__device__ __forceinline__ void patch_constraints(const XpbdWorld& W, const XpbdDevParams& P, const XpbdPatch& pt,
                                                  const PatchView& v, const float4* __restrict__ spos,
                                                  float4* __restrict__ sres, TailMode tail) {
    const float* pal = W.palette_comp + (uint32_t)pt.cloth * XPBD_PALETTE;
    const bool persist = P.lambda_mode != 0u;
#pragma unroll 2
    for (uint32_t c = threadIdx.x; c < pt.nc; c += blockDim.x) {
        const uint2 rec = v.con[c];
        const float4 pi = spos[rec.x & 0xFFFu], pj = spos[(rec.x >> 12) & 0xFFFu];
        const F3 gv = sub3(f3(pi), f3(pj));
        const float len = len3(gv);
        float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
        bool reset_lam = persist && tail == kTailFinalizePredict;
        if (!(len < 1e-8f)) {
            const F3 nrm = div3(gv, len);
            const float C = __fsub_rn(len, __uint_as_float(rec.y));
            const float alpha_t = __fmul_rn(pal[(rec.x >> 24) & 0xFu], P.inv_dt_sq);
            const float wsum = __fadd_rn(__fadd_rn(pi.w, pj.w), alpha_t);
            float dlam = 0.0f;
            if (!(wsum < 1e-8f)) {
                const float lam = persist ? W.patch_lambda[pt.lam_off + c] : 0.0f;
                dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, lam)), wsum);
                if (persist) {
                    W.patch_lambda[pt.lam_off + c] = reset_lam ? 0.0f : __fadd_rn(lam, dlam);
                    reset_lam = false;
                }
            }
            r = make_float4(nrm.x, nrm.y, nrm.z, dlam);
        }
        if (reset_lam) W.patch_lambda[pt.lam_off + c] = 0.0f;
        sres[c] = r;
    }
}

__device__ __forceinline__ void patch_gather(const XpbdWorld& W, const XpbdDevParams& P, const XpbdPatch& pt,
                                             const PatchView& v, const float4* spos, const float4* sres,
                                             float4* __restrict__ jout, TailMode tail) {
    for (uint32_t k = threadIdx.x; k < pt.np; k += blockDim.x) {
        const float4 ps = spos[k];
        if (ps.w <= 0.0f) continue;  // pinned: both buffers already hold the fixed position
        const uint32_t q0 = v.gofs[k], q1 = v.gofs[k + 1];
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        for (uint32_t q = q0; q < q1; ++q) {
            const uint32_t sl = v.slots[q];
            const float4 r = sres[sl & 0x7FFFu];
            const bool neg = (sl & 0x8000u) != 0u;
            ax = __fadd_rn(ax, __fmul_rn(__fmul_rn(neg ? -r.x : r.x, ps.w), r.w));
            ay = __fadd_rn(ay, __fmul_rn(__fmul_rn(neg ? -r.y : r.y, ps.w), r.w));
            az = __fadd_rn(az, __fmul_rn(__fmul_rn(neg ? -r.z : r.z, ps.w), r.w));
        }
        F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
        if (P.relaxation == 1u && q1 > q0) delta = div3(delta, (float)(q1 - q0));
        delta = clamp_correction(delta);
        F3 xn = add3(f3(ps), delta);
        const uint32_t g = v.parts[k];
        if (tail == kTailNone) {
            jout[g] = make_float4(xn.x, xn.y, xn.z, ps.w);
            continue;
        }
        const F3 xo = f3(W.x[g]);
        F3 vel = f3(W.v[g]);
        xn = finalize_particle(xn, xo, vel, P, W.status);
        W.x[g] = make_float4(xn.x, xn.y, xn.z, ps.w);
        W.v[g] = make_float4(vel.x, vel.y, vel.z, 0.0f);
        if (tail == kTailFinalizePredict) {
            const F3 pos = predict_w(W, g, xn, vel, P);
            jout[g] = make_float4(pos.x, pos.y, pos.z, ps.w);
        } else {
            jout[g] = make_float4(xn.x, xn.y, xn.z, ps.w);
        }
    }
}

// Persistent Jacobi over spatial patches; same flags / buffer protocol as jacobi_persistent_kernel. Shared memory:
// two blob buffers, two particle buffers, one constraint-result buffer, two mbarriers.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) jacobi_patch_kernel(XpbdWorld W, uint32_t flags, uint32_t substeps,
                                                             uint32_t pend, uint32_t start) {
    extern __shared__ __align__(128) unsigned char s_dyn[];
    if (!status_clear(W)) return;
    const XpbdDevParams P = *W.params;
    const bool persist = P.lambda_mode != 0u;
    unsigned char* blob[2] = {s_dyn, s_dyn + W.patch_max_blob};
    float4* spos[2] = {reinterpret_cast<float4*>(s_dyn + 2 * W.patch_max_blob),
                       reinterpret_cast<float4*>(s_dyn + 2 * W.patch_max_blob) + W.patch_max_local};
    float4* sres = spos[1] + W.patch_max_local;
    uint64_t* bars = reinterpret_cast<uint64_t*>(sres + W.patch_max_con);
    if (threadIdx.x == 0) {
        mbar_init1(&bars[0]);
        mbar_init1(&bars[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t phase[2] = {0u, 0u};
    bool inflight[2] = {false, false};                   // issued and not yet waited for
    uint32_t bsel = 0;                                   // blob buffer of the current patch
    const uint32_t mine = W.n_patches > blockIdx.x ? (W.n_patches - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    auto issue_blob = [&](uint32_t m, uint32_t b) {      // my m-th patch (of any iteration) into buffer b
        const XpbdPatch& pt = W.patches[blockIdx.x + (m % mine) * gridDim.x];
        if (threadIdx.x == 0) bulk_g2s_evict_first(blob[b], W.patch_blob + pt.off16, pt.bytes, &bars[b]);
        inflight[b] = true;
    };
    bool failed = false;
    auto wait_blob = [&](uint32_t b) {
        if (!mbar_wait_bounded(&bars[b], phase[b])) {
            failed = true;
            if (threadIdx.x == 0) set_status(W.status, XPBD_DEV_BARRIER_TIMEOUT);
        }
        inflight[b] = false;
    };
    if (mine > 0 && (*W.params).iterations > 0 && substeps > 0) issue_blob(0, 0);

    predict_phase(W, P, (flags & kBeginFinalize) != 0u, pend, start, true);
    if (persist) {  // λ of every patch constraint slot starts the substep at zero
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < W.patch_con_total; k += stride)
            W.patch_lambda[k] = 0.0f;
    }
    bool ok = grid_barrier(W, P);
    uint32_t b = start;
    const uint32_t I = P.iterations;
    uint32_t seq = 0;  // running index of my processed patches (blob pipeline position)
    for (uint32_t s = 0; s < substeps && ok; ++s) {
        const bool last_sub = (s + 1 == substeps);
        if (I == 0) {
            const uint32_t stride = gridDim.x * blockDim.x;
            const bool fin = !last_sub || (flags & kEndFinalize);
            for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n && fin; i += stride) {
                float4 p4 = W.jac[b][i];
                if (p4.w <= 0.0f) continue;
                const F3 xo = f3(W.x[i]);
                F3 vel = f3(W.v[i]);
                F3 xn = finalize_particle(f3(p4), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                if (!last_sub) {
                    F3 pos = predict_w(W, i, xn, vel, P);
                    W.jac[b][i] = make_float4(pos.x, pos.y, pos.z, p4.w);
                }
            }
            if (!last_sub) ok = grid_barrier(W, P);
            continue;
        }
        for (uint32_t k = 0; k < I && ok; ++k) {
            const float4* jin = W.jac[(b + k) & 1u];
            float4* jout = W.jac[(b + k + 1) & 1u];
            TailMode tail = kTailNone;
            if (k + 1 == I) {
                if (!last_sub) tail = kTailFinalizePredict;
                else if (flags & kEndFinalize) tail = kTailFinalize;
            }
            const bool very_last = last_sub && (k + 1 == I);
            uint32_t ps = 0;
            for (uint32_t m = 0; m < mine && !failed; ++m, ++seq) {
                const XpbdPatch pt = W.patches[blockIdx.x + m * gridDim.x];
                const uint32_t nl = (uint32_t)pt.np + pt.nh;
                wait_blob(bsel);
                phase[bsel] ^= 1u;
                const PatchView v = patch_view(blob[bsel], pt);
                // the next patch's blob (also across the iteration boundary; not after the launch's last patch)
                const bool more = (m + 1 < mine) || !very_last;
                if (more) issue_blob(seq + 1, bsel ^ 1u);
                if (m == 0) {
                    for (uint32_t t = threadIdx.x; t < nl; t += blockDim.x) spos[ps][t] = jin[v.parts[t]];
                } else {
                    cp_async_wait_all();
                }
                __syncthreads();
                patch_constraints(W, P, pt, v, spos[ps], sres, tail);
                __syncthreads();
                if (m + 1 < mine) {  // gather the next patch's particles while this one finishes
                    const XpbdPatch pn = W.patches[blockIdx.x + (m + 1) * gridDim.x];
                    wait_blob(bsel ^ 1u);
                    const PatchView vn = patch_view(blob[bsel ^ 1u], pn);
                    const uint32_t nln = (uint32_t)pn.np + pn.nh;
                    for (uint32_t t = threadIdx.x; t < nln; t += blockDim.x) cp_async16(&spos[ps ^ 1u][t], jin + vn.parts[t]);
                    cp_async_commit();
                }
                patch_gather(W, P, pt, v, spos[ps], sres, jout, tail);
                __syncthreads();
                bsel ^= 1u;
                ps ^= 1u;
            }
            if (failed) break;
            if (!very_last) ok = grid_barrier(W, P);
        }
        b = (b + I) & 1u;
    }
    // no copy may still target this CTA's shared memory when it exits (bounded waits)
    for (uint32_t q = 0; q < 2; ++q)
        if (inflight[q]) mbar_wait_bounded(&bars[q], phase[q]);
    cp_async_wait_all();
}

// ---------------------------------------------------------------------------------------------- Gauss–Seidel
// One constraint of the colored sweep, xpbd_cpu.rs:349-385, in place on the working state.
__device__ __forceinline__ void gs_constraint(const XpbdWorld& W, const XpbdDevParams& P, uint32_t e, float4* jw,
                                              bool persist) {
    const uint4 c = W.con[e];
    const uint32_t i = c.x, j = c.y;
    const float4 pi4 = jw[i];
    const float4 pj4 = jw[j];
    const float w_i = pi4.w, w_j = pj4.w;
    if (w_j <= 0.0f && w_i <= 0.0f) return;
    const F3 p_i = f3(pi4), p_j = f3(pj4);
    F3 gv = sub3(p_i, p_j);
    const float len = len3(gv);
    if (len < 1e-8f) return;
    gv = div3(gv, len);
    const float C = __fsub_rn(len, __uint_as_float(c.z));
    const float alpha_t = __fmul_rn(__uint_as_float(c.w), P.inv_dt_sq);
    const float wsum = __fadd_rn(__fadd_rn(w_i, w_j), alpha_t);
    if (wsum < 1e-8f) return;
    const float lam = persist ? W.con_lambda[e] : 0.0f;
    const float dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, lam)), wsum);
    if (persist) W.con_lambda[e] = __fadd_rn(lam, dlam);
    const F3 og = {__fmul_rn(P.omega, gv.x), __fmul_rn(P.omega, gv.y), __fmul_rn(P.omega, gv.z)};
    const F3 dx_i = clamp_correction(mul3(mul3(og, w_i), dlam));
    const F3 dx_j = clamp_correction(neg3(mul3(mul3(og, w_j), dlam)));
    if (w_i > 0.0f) {
        const F3 n = add3(p_i, dx_i);
        jw[i] = make_float4(n.x, n.y, n.z, w_i);
    }
    if (w_j > 0.0f) {
        const F3 n = add3(p_j, dx_j);
        jw[j] = make_float4(n.x, n.y, n.z, w_j);
    }
}

// Persistent colored Gauss–Seidel: per inner iteration one sweep over the color batches, a grid barrier after each
// color (colors are particle-disjoint, so a color's constraints run in parallel with the reference's result).
// The working state is jac[0]; with kBeginFinalize the first substep finalizes positions waiting in jac[pend].
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) gs_persistent_kernel(XpbdWorld W, uint32_t flags, uint32_t substeps,
                                                              uint32_t pend) {
    if (!status_clear(W)) return;
    const XpbdDevParams P = *W.params;
    const bool persist = P.lambda_mode != 0u;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gstride = gridDim.x * blockDim.x;
    float4* jw = W.jac[0];
    bool pending = (flags & kBeginFinalize) != 0u;
    for (uint32_t s = 0; s < substeps; ++s) {
        predict_phase(W, P, pending, s == 0 ? pend : 0u, 0, true);
        if (persist)
            for (uint32_t e = gtid; e < W.e; e += gstride) W.con_lambda[e] = 0.0f;
        if (!grid_barrier(W, P)) return;
        for (uint32_t k = 0; k < P.iterations; ++k)
            for (uint32_t c = 0; c < W.n_colors; ++c) {
                const uint32_t e0 = W.color_off[c], e1 = W.color_off[c + 1];
                for (uint32_t e = e0 + gtid; e < e1; e += gstride) gs_constraint(W, P, e, jw, persist);
                if (!grid_barrier(W, P)) return;
            }
        pending = true;
    }
    if (flags & kEndFinalize) predict_phase(W, P, true, 0, 0, false);
}

// Standalone finalize of positions waiting in jac[pend] (after a collision pass on the last substep).
__global__ void finalize_kernel(XpbdWorld W, uint32_t pend) {
    const XpbdDevParams P = *W.params;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n; i += stride) {
        float4 p4 = W.jac[pend][i];
        if (p4.w <= 0.0f) continue;
        const F3 xo = f3(W.x[i]);
        F3 vel = f3(W.v[i]);
        F3 xn = finalize_particle(f3(p4), xo, vel, P, W.status);
        W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
        W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
    }
}

// Max strain residual over constraints [e0, e1) of the input-order table (non-negative floats compare as ints).
__global__ void strain_residual_kernel(XpbdWorld W, uint32_t e0, uint32_t e1, unsigned* out_bits) {
    float m = 0.0f;
    for (uint32_t e = e0 + blockIdx.x * blockDim.x + threadIdx.x; e < e1; e += gridDim.x * blockDim.x) {
        const uint4 c = W.con_in[e];
        const float len = len3(sub3(f3(W.x[c.x]), f3(W.x[c.y])));
        const float rest = __uint_as_float(c.z);
        const float s = fabsf(__fsub_rn(len, rest)) / rest;
        m = fmaxf(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(kFull, m, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(out_bits, __float_as_uint(m));
}

// ---------------------------------------------------------------------------------------------- host launchers
template <int BLOCK>
static const void* jacobi_fn() { return (const void*)jacobi_persistent_kernel<BLOCK>; }
template <int BLOCK>
static const void* patch_fn() { return (const void*)jacobi_patch_kernel<BLOCK>; }
template <int BLOCK>
static const void* row_fn() { return (const void*)jacobi_row_kernel<BLOCK>; }

template <int BLOCK>
static const void* converge_fn() { return (const void*)jacobi_converge_kernel<BLOCK>; }
template <int BLOCK>
static const void* gs_fn() { return (const void*)gs_persistent_kernel<BLOCK>; }

// kernel 0: Jacobi over warp tiles, 1: Gauss–Seidel, 2: Jacobi over spatial patches, 5: Jacobi thread per particle,
// 6: convergence solve
const void* solver_kernel_fn(uint32_t solver, uint32_t block) {
    switch (solver * 10000 + block) {
        case 128: return jacobi_fn<128>();
        case 256: return jacobi_fn<256>();
        case 512: return jacobi_fn<512>();
        case 1024: return jacobi_fn<1024>();
        case 10128: return gs_fn<128>();
        case 10256: return gs_fn<256>();
        case 10512: return gs_fn<512>();
        case 11024: return gs_fn<1024>();
        case 20128: return patch_fn<128>();
        case 20256: return patch_fn<256>();
        case 20512: return patch_fn<512>();
        case 21024: return patch_fn<1024>();
        case 50128: return row_fn<128>();
        case 50256: return row_fn<256>();
        case 50512: return row_fn<512>();
        case 51024: return row_fn<1024>();
        case 60128: return converge_fn<128>();
        case 60256: return converge_fn<256>();
        case 60512: return converge_fn<512>();
        case 61024: return converge_fn<1024>();

    }
    return nullptr;
}

static size_t solver_dyn_smem(uint32_t solver, uint32_t block, const XpbdWorld& W) {
    if (solver == 0) return (size_t)(block / 32) * 3 * kTileChunk * sizeof(float);
    if (solver == 2)
        return 2 * (size_t)W.patch_max_blob + (2 * (size_t)W.patch_max_local + W.patch_max_con) * sizeof(float4) + 16;
    return 0;
}

// Opt in to the dynamic shared memory explicitly: the default 48 KB limit covers static + dynamic together.
static bool set_smem_attr(const void* fn, size_t dyn) {
    if (dyn == 0) return true;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) == cudaSuccess;
}

cudaError_t launch_solver(uint32_t solver, uint32_t block, uint32_t grid, bool cooperative, const XpbdWorld& W,
                          uint32_t flags, uint32_t substeps, uint32_t pend, uint32_t start, cudaStream_t st) {
    const void* fn = solver_kernel_fn(solver, block);
    if (!fn) return cudaErrorInvalidValue;
    const size_t dyn = solver_dyn_smem(solver, block, W);
    if (!set_smem_attr(fn, dyn)) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    if (cooperative) {
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    XpbdWorld w = W;
    if (solver == 6) {  // convergence solve: `flags` carries the warm-start switch
        void* args[] = {&w, &flags};
        return cudaLaunchKernelExC(&cfg, fn, args);
    }
    if (solver != 1) {
        void* args[] = {&w, &flags, &substeps, &pend, &start};
        return cudaLaunchKernelExC(&cfg, fn, args);
    }
    void* args[] = {&w, &flags, &substeps, &pend};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

int max_blocks_per_sm(uint32_t solver, uint32_t block, const XpbdWorld& W) {
    const void* fn = solver_kernel_fn(solver, block);
    const size_t dyn = solver_dyn_smem(solver, block, W);
    int nb = 0;
    if (!fn || !set_smem_attr(fn, dyn)) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, (int)block, dyn) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_converge_predict(const XpbdWorld& W, int sms, cudaStream_t st) {
    uint32_t grid = (W.n + 255) / 256;
    if (grid > (uint32_t)sms * 8) grid = (uint32_t)sms * 8;
    if (grid < 16) grid = 16;
    converge_predict_kernel<<<grid, 256, 0, st>>>(W);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const XpbdWorld& W, uint32_t pend, int sms, cudaStream_t st) {
    uint32_t grid = (W.n + 255) / 256;
    if (grid > (uint32_t)sms * 8) grid = (uint32_t)sms * 8;
    if (grid == 0) grid = 1;
    finalize_kernel<<<grid, 256, 0, st>>>(W, pend);
    return cudaGetLastError();
}

cudaError_t launch_strain_residual(const XpbdWorld& W, uint32_t e0, uint32_t e1, unsigned* out_bits, int sms,
                                   cudaStream_t st) {
    uint32_t n = e1 - e0;
    uint32_t grid = (n + 255) / 256;
    if (grid > (uint32_t)sms * 4) grid = (uint32_t)sms * 4;
    if (grid == 0) grid = 1;
    strain_residual_kernel<<<grid, 256, 0, st>>>(W, e0, e1, out_bits);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- vertex normals
// accumulate_normals + finalize_normals (cloth_sim_jacobi.wgsl:492-547): per triangle c = cross(p1 - p0, p2 - p0),
// converted to fixed point i32(c · 33333) (round toward zero, saturating) and summed into each of its three vertices;
// then n = f32(sum) / 33333, normalised when |n| > 1e-8, else (0, 1, 0). The reference sums with integer atomics; here
// each vertex gathers its triangles from a vertex → triangle table (no atomics). Integer sums (wrapping, as i32
// atomics wrap) do not depend on order, so the result is the same bits either way.
__device__ __forceinline__ int fixed_normal(float c) { return __float2int_rz(__fmul_rn(c, 33333.0f)); }

__global__ void vertex_normals_kernel(XpbdWorld W) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < W.n; v += gridDim.x * blockDim.x) {
        uint32_t sx = 0u, sy = 0u, sz = 0u;  // i32 sums with wrap-around
        for (uint32_t k = W.vt_off[v]; k < W.vt_off[v + 1]; ++k) {
            const uint4 t = W.tris[W.vt_tri[k]];
            const F3 p0 = f3(W.x[t.x]), p1 = f3(W.x[t.y]), p2 = f3(W.x[t.z]);
            const F3 e0 = sub3(p1, p0), e1 = sub3(p2, p0);
            const float cx = __fsub_rn(__fmul_rn(e0.y, e1.z), __fmul_rn(e0.z, e1.y));
            const float cy = __fsub_rn(__fmul_rn(e0.z, e1.x), __fmul_rn(e0.x, e1.z));
            const float cz = __fsub_rn(__fmul_rn(e0.x, e1.y), __fmul_rn(e0.y, e1.x));
            sx += (uint32_t)fixed_normal(cx);
            sy += (uint32_t)fixed_normal(cy);
            sz += (uint32_t)fixed_normal(cz);
        }
        F3 n = {__fdiv_rn(__int2float_rn((int)sx), 33333.0f), __fdiv_rn(__int2float_rn((int)sy), 33333.0f),
                __fdiv_rn(__int2float_rn((int)sz), 33333.0f)};
        const float ln = len3(n);
        n = (ln > 1e-8f) ? div3(n, ln) : F3{0.0f, 1.0f, 0.0f};
        W.normals[v] = make_float4(n.x, n.y, n.z, 0.0f);
    }
}

cudaError_t launch_vertex_normals(const XpbdWorld& W, int sms, cudaStream_t st) {
    uint32_t grid = (W.n + 255) / 256;
    if (grid > (uint32_t)sms * 8) grid = (uint32_t)sms * 8;
    if (grid == 0) grid = 1;
    vertex_normals_kernel<<<grid, 256, 0, st>>>(W);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- self test
// The shared-reciprocal division against the ordinary correctly rounded division on `count` operand triples drawn
// (splitmix64 of the index) over all finite float bit patterns for the numerators and for the divisor.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float finite_bits(uint32_t u) {
    const float f = __uint_as_float(u);
    return isfinite(f) ? f : __uint_as_float(u & 0xBF7FFFFFu);  // clear an exponent bit: finite
}
__global__ void division_selftest_kernel(uint64_t count, uint64_t seed, unsigned long long* mismatches) {
    unsigned long long bad = 0;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < count;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r0 = splitmix64(seed ^ (2 * k)), r1 = splitmix64(seed ^ (2 * k + 1));
        float ax = finite_bits((uint32_t)r0), ay = finite_bits((uint32_t)(r0 >> 32)), az = finite_bits((uint32_t)r1);
        float b = finite_bits((uint32_t)(r1 >> 32));
        // half the samples: operands of a cloth step (differences of nearby positions over their length)
        if (k & 1ull) {
            b = fabsf(b);
            const float e = __uint_as_float(0x3F800000u | ((uint32_t)r1 & 0x7FFFFFu));  // [1, 2)
            b = __fmul_rn(e, __uint_as_float((uint32_t)(((r1 >> 23) % 60u) + 97u) << 23));  // ~1e-9 .. 1e9
            ax = __fmul_rn(b, __fmul_rn(__uint_as_float(0x3F800000u | ((uint32_t)r0 & 0x7FFFFFu)), -0.7f));
            ay = __fmul_rn(b, __uint_as_float((uint32_t)(r0 >> 40) | 0x3E000000u));
            if ((k & 6ull) == 2ull) az = 0.0f;                                        // exact zero component
            if ((k & 6ull) == 4ull) az = __fmul_rn(az, 0x1p-100f);                      // tiny component
        }
        float qx, qy, qz;
        fpdiv3(ax, ay, az, b, qx, qy, qz);
        float rx = __fdiv_rn(ax, b), ry = __fdiv_rn(ay, b), rz = __fdiv_rn(az, b);
        bad += (__float_as_uint(qx) != __float_as_uint(rx) && !(isnan(qx) && isnan(rx)));
        bad += (__float_as_uint(qy) != __float_as_uint(ry) && !(isnan(qy) && isnan(ry)));
        bad += (__float_as_uint(qz) != __float_as_uint(rz) && !(isnan(qz) && isnan(rz)));
        // a vector over its own correctly rounded length: where the fast path reports success it must be exact
        {
            const float len = len3(F3{ax, ay, az});
            if (fpdiv3_by_length_fast(ax, ay, az, len, qx, qy, qz)) {
                rx = __fdiv_rn(ax, len);
                ry = __fdiv_rn(ay, len);
                rz = __fdiv_rn(az, len);
                bad += (__float_as_uint(qx) != __float_as_uint(rx));
                bad += (__float_as_uint(qy) != __float_as_uint(ry));
                bad += (__float_as_uint(qz) != __float_as_uint(rz));
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) bad += __shfl_xor_sync(kFull, bad, o);
    if ((threadIdx.x & 31u) == 0 && bad) atomicAdd(mismatches, bad);
}
cudaError_t launch_division_selftest(uint64_t count, uint64_t seed, unsigned long long* mismatches, int sms,
                                     cudaStream_t st) {
    division_selftest_kernel<<<sms * 8, 256, 0, st>>>(count, seed, mismatches);
    return cudaGetLastError();
}

}  // namespace xpbd
