// Colored Gauss–Seidel for a sheet that fits in one thread-block cluster (sm_100a distributed shared memory).
//
// Same arithmetic as the grid-wide solver (gs_constraint, xpbd_cpu.rs:349-385; WGSL gs_edges,
// cloth_sim.wgsl:154-210), different execution. A cluster of CL CTAs (8 portable or 16 non-portable) keeps the whole
// working state — every particle as float4 {x, y, z, inverse mass} — in distributed shared memory: CTA r owns
// particles [r*P, (r+1)*P) with P a power of two, local particle p in slot cluster_slot(p). A color batch is split by
// the CTA owning its first endpoint; each CTA streams its chunk of constraint records from global memory into shared
// memory with a TMA bulk copy (cp.async.bulk, completion on an mbarrier), double-buffered so the next color's chunk
// lands while the current one is solved, and reads/writes both endpoints through shared::cluster loads and stores.
// Colors are separated by the hardware cluster barrier (barrier.cluster arrive.release / wait.acquire) instead of a
// global-memory grid barrier.
// Every CTA executes the same barrier sequence (no early exit); mbarrier waits are bounded and report
// XPBD_DEV_BARRIER_TIMEOUT if exceeded.
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "xpbd_cluster.h"
#include "xpbd_fpdiv.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {

namespace {

constexpr float kCap = 0.28f;     // JACOBI_CORRECTION_CAP
constexpr float kVmax = 12.0f;    // PREDICT_MAX_SPEED
constexpr float kGrab = 0.065f;   // GRAB_MAX_PULL_PER_SUBSTEP

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 vmul(V3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ V3 vdiv(V3 a, float s) {  // correctly rounded, one shared reciprocal (xpbd_fpdiv.h)
    V3 q;
    fpdiv3(a.x, a.y, a.z, s, q.x, q.y, q.z);
    return q;
}
__device__ __forceinline__ float vlen(V3 a) {
    return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z)));
}
// clamp_correction (xpbd_cpu.rs:28-36), skipping the root when |dx|² <= the largest float not above 0.28f².
__device__ __forceinline__ V3 vclamp(V3 dx) {
    const float d = __fadd_rn(__fadd_rn(__fmul_rn(dx.x, dx.x), __fmul_rn(dx.y, dx.y)), __fmul_rn(dx.z, dx.z));
    if (d <= __uint_as_float(0x3da0902du)) return dx;
    const float ml = __fsqrt_rn(d);
    if (ml > kCap && ml > 0.0f) return vmul(dx, __fdiv_rn(kCap, ml));
    return dx;
}
// vclamp of dx = RN(RN(og·w)·dlam) with og = RN(ω·n̂), given bound = RN(RN(ω·w)·dlam): |n̂| <= 1 + 2^-22 (each
// component a correctly rounded quotient by a length rounded at most 2.5 ulp low), so |dx| <= |bound|·(1 + 2^-20);
// when |bound| <= 0.27 the rounded |dx|² is below 0.0730 and the reference's clamp (|dx|² > 0.28²,
// xpbd_cpu.rs:28-36) cannot apply, which skips the squared length. NaN or larger bounds take the full test.
__device__ __forceinline__ V3 vclamp_bounded(V3 dx, float bound) {
    if (fabsf(bound) <= 0.27f) return dx;
    return vclamp(dx);
}
__device__ __forceinline__ bool vfinite(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

__device__ __forceinline__ V3 predict(uint32_t i, V3 sim, V3& vel, const XpbdDevParams& P, const XpbdWorld& W) {
    V3 v = vadd(vel, vmul(V3{P.gravity[0], P.gravity[1], P.gravity[2]}, P.dt));
    if (*W.wind_count != 0u) {  // per-cloth wind (extension): v += (wind − v) · (drag · dt)
        const XpbdWind wd = W.winds[W.row_cloth[i]];
        if (wd.drag > 0.0f) v = vadd(v, vmul(vsub(V3{wd.vel[0], wd.vel[1], wd.vel[2]}, v), __fmul_rn(wd.drag, P.dt)));
    }
    const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(v.x, v.x), __fmul_rn(v.y, v.y)), __fmul_rn(v.z, v.z));
    if (v2 >= 144.0f) {
        const float speed = __fsqrt_rn(v2);
        if (speed > kVmax && speed > 0.0f) v = vmul(v, __fdiv_rn(kVmax, speed));
    }
    V3 pos = vadd(sim, vmul(v, P.dt));
    if (P.grab_active != 0u && (int32_t)i == P.grab_idx) {
        V3 pull = vmul(vsub(V3{P.grab_target[0], P.grab_target[1], P.grab_target[2]}, pos), P.grab_stiffness);
        const float pl = vlen(pull);
        if (pl > kGrab && pl > 0.0f) pull = vmul(pull, __fdiv_rn(kGrab, pl));
        pos = vadd(pos, pull);
    }
    vel = v;
    return pos;
}

__device__ __forceinline__ V3 finalize(V3 xn, V3 xo, V3& vel, const XpbdDevParams& P, int* status) {
    if (P.ground_enabled != 0u && xn.y < P.ground_y) xn.y = P.ground_y;
    vel = vmul(vmul(vsub(xn, xo), P.inv_dt), P.damp);
    if (!vfinite(xn) || !vfinite(vel)) atomicOr(status, XPBD_DEV_NONFINITE);
    return xn;
}

// ---- PTX wrappers: mbarrier + bulk copy (cluster rank, DSMEM and the cluster barrier: xpbd_cluster.h)
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
// Bounded wait for phase `parity` of `bar`; false if the limit was reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
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

// One constraint of the reference's colored sweep (xpbd_cpu.rs:312-391): both endpoints move by their clamped
// corrections, pinned endpoints stay.
// Endpoint i is always this CTA's particle (records are grouped by the rank owning i) and goes through the CTA's own
// shared window (xs_base); endpoint j too for interior records (LOCAL), otherwise through the cluster window of the
// CTA owning it.
// PLAIN (XpbdDevParams::plain_terms): α̃ finite, so −C − α̃·0 = −C, and a constraint with a free endpoint has a w sum
// >= 1e-8 (constraints between two pinned particles return before), so the w-sum test is skipped.
template <bool LOCAL, bool PLAIN>
__device__ __forceinline__ void gs_solve(const uint4 cr, const uint32_t* s_rank_base, uint32_t xs_base, uint32_t shift,
                                         uint32_t mask, const XpbdDevParams& P) {
    const uint32_t ai = xs_base + ((cr.x & mask) << 4);
    const uint32_t aj = (LOCAL ? xs_base : s_rank_base[cr.y >> shift]) + ((cr.y & mask) << 4);
    const float4 pi4 = ld_local(ai);
    const float4 pj4 = LOCAL ? ld_local(aj) : ld_dsmem(aj);
    const float w_i = pi4.w, w_j = pj4.w;
    if (w_j <= 0.0f && w_i <= 0.0f) return;
    const V3 p_i = v3(pi4), p_j = v3(pj4);
    V3 gv = vsub(p_i, p_j);
    const float len = vlen(gv);
    if (len < 1e-8f) return;
    {
        V3 q;
        if (!fpdiv3_by_length_fast(gv.x, gv.y, gv.z, len, q.x, q.y, q.z)) q = vdiv(gv, len);
        gv = q;
    }
    const float C = __fsub_rn(len, __uint_as_float(cr.z));
    const float alpha_t = __fmul_rn(__uint_as_float(cr.w), P.inv_dt_sq);
    const float wsum = __fadd_rn(__fadd_rn(w_i, w_j), alpha_t);
    if (!PLAIN && wsum < 1e-8f) return;
    const float dlam = __fdiv_rn(PLAIN ? -C : __fsub_rn(-C, __fmul_rn(alpha_t, 0.0f)), wsum);
    const V3 og = {__fmul_rn(P.omega, gv.x), __fmul_rn(P.omega, gv.y), __fmul_rn(P.omega, gv.z)};
    const V3 dx_i = vclamp_bounded(vmul(vmul(og, w_i), dlam), __fmul_rn(__fmul_rn(P.omega, w_i), dlam));
    V3 dxj = vmul(vmul(og, w_j), dlam);
    const V3 dx_j = vclamp_bounded(V3{-dxj.x, -dxj.y, -dxj.z}, __fmul_rn(__fmul_rn(P.omega, w_j), dlam));
    if (w_i > 0.0f) {
        const V3 n = vadd(p_i, dx_i);
        st_local(ai, make_float4(n.x, n.y, n.z, w_i));
    }
    if (w_j > 0.0f) {
        const V3 n = vadd(p_j, dx_j);
        if (LOCAL)
            st_local(aj, make_float4(n.x, n.y, n.z, w_j));
        else
            st_dsmem(aj, make_float4(n.x, n.y, n.z, w_j));
    }
}

}  // namespace

// T.off[(c * CL + r)] .. T.off[c * CL + r + 1]: records of color c owned by rank r (uint4 {i, j, rest, comp}, the
// endpoints as rank << shift | shared-memory slot).
template <int CL>
__global__ void __launch_bounds__(1024, 1) gs_cluster_kernel(XpbdWorld W, ClusterTable T, uint32_t flags,
                                                              uint32_t substeps, uint32_t pend) {
    extern __shared__ __align__(128) unsigned char smem[];
    const XpbdDevParams P = *W.params;
    const uint32_t rank = cluster_rank();
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t shift = T.shift, mask = (1u << T.shift) - 1u;
    const uint32_t base = rank << shift;
    const uint32_t cnt = base < W.n ? min(1u << shift, W.n - base) : 0u;
    float4* xs = reinterpret_cast<float4*>(smem);
    uint4* buf0 = reinterpret_cast<uint4*>(smem + ((size_t)16 << shift));
    uint4* buf1 = buf0 + T.max_chunk;
    uint64_t* bars = reinterpret_cast<uint64_t*>(buf1 + T.max_chunk);
    __shared__ uint32_t s_rank_base[16];
    const uint32_t xs_base = smem_u32(xs);
    if (tid < CL) s_rank_base[tid] = map_rank(smem_u32(xs), tid);
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    bool failed = false;
    const uint32_t ncol = W.n_colors;
    const uint32_t I = P.iterations;
    // chunk schedule: q = 0, 1, 2, ... over (substep, iteration, color); chunk q uses buffer q&1
    uint32_t phase[2] = {0u, 0u};
    // the group offsets are read every sweep: keep them in shared memory when they fit
    constexpr uint32_t kMaxCachedGroups = 512;
    __shared__ uint32_t s_off[kMaxCachedGroups + 1], s_nbd[kMaxCachedGroups];
    const bool cached = ncol * CL <= kMaxCachedGroups;
    if (cached) {
        for (uint32_t k = tid; k <= ncol * CL; k += nthr) s_off[k] = T.off[k];
        for (uint32_t k = tid; k < ncol * CL; k += nthr) s_nbd[k] = T.nbd[k];
    }
    __syncthreads();
    auto chunk_range = [&](uint32_t c, uint32_t& e0, uint32_t& e1) {
        e0 = cached ? s_off[c * CL + rank] : T.off[c * CL + rank];
        e1 = cached ? s_off[c * CL + rank + 1] : T.off[c * CL + rank + 1];
    };
    auto issue = [&](uint32_t c, uint32_t b) {
        uint32_t e0, e1;
        chunk_range(c, e0, e1);
        if (tid == 0 && e1 > e0) bulk_load(b ? buf1 : buf0, T.rec + e0, (e1 - e0) * 16u, &bars[b]);
    };
    const uint32_t total_chunks = substeps * I * ncol;
    bool pending = (flags & kBeginFinalize) != 0u;
    if (total_chunks > 0) issue(0, 0);
    uint32_t q = 0;
    for (uint32_t s = 0; s < substeps; ++s) {
        // predict (own particles): optionally finalize the pending result first
        for (uint32_t k = tid; k < cnt; k += nthr) {
            const uint32_t i = base + k;
            const float4 x4 = W.x[i];
            if (x4.w <= 0.0f) {
                xs[cluster_slot(k)] = x4;
                continue;
            }
            V3 xo = v3(x4);
            V3 vel = v3(W.v[i]);
            if (pending) {
                const V3 xn = finalize(v3(W.jac[s == 0 ? pend : 0u][i]), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, x4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                xo = xn;
            }
            V3 p = predict(i, xo, vel, P, W);
            if (*W.grab_count != 0u) {  // per-cloth grab (extension), the reference's pull on the grabbed vertex
                const XpbdGrab g = W.grabs[W.row_cloth[i]];
                if (g.idx == (int32_t)i) {
                    V3 pull = vmul(vsub(V3{g.target[0], g.target[1], g.target[2]}, p), g.stiffness);
                    const float pl = vlen(pull);
                    if (pl > kGrab && pl > 0.0f) pull = vmul(pull, __fdiv_rn(kGrab, pl));
                    p = vadd(p, pull);
                }
            }
            xs[cluster_slot(k)] = make_float4(p.x, p.y, p.z, x4.w);
        }
        pending = true;
        cluster_sync();
        for (uint32_t it = 0; it < I; ++it) {
            for (uint32_t c = 0; c < ncol; ++c, ++q) {
                const uint32_t b = q & 1u;
                if (q + 1 < total_chunks) issue((c + 1) % ncol, b ^ 1u);  // prefetch the next color's chunk
                uint32_t e0, e1;
                chunk_range(c, e0, e1);
                const uint32_t nb = cached ? s_nbd[c * CL + rank] : T.nbd[c * CL + rank];
                const uint4* rec = b ? buf1 : buf0;
                if (e1 > e0) {
                    if (!mbar_wait(&bars[b], phase[b])) {
                        failed = true;
                        if (tid == 0) atomicOr(W.status, XPBD_DEV_BARRIER_TIMEOUT);
                    }
                    phase[b] ^= 1u;
                }
                // records touching boundary particles, then the cluster barrier's arrive, then the records of this
                // CTA's interior particles (no other CTA reads or writes those) while the barrier completes
                auto sweep = [&](auto plain_tag) {
                    constexpr bool PL = decltype(plain_tag)::value;
                    for (uint32_t e = tid; e < nb && !failed; e += nthr)
                        gs_solve<false, PL>(rec[e], s_rank_base, xs_base, shift, mask, P);
                    cluster_arrive();
                    for (uint32_t e = nb + tid; e < e1 - e0 && !failed; e += nthr)
                        gs_solve<true, PL>(rec[e], s_rank_base, xs_base, shift, mask, P);
                };
                if (P.plain_terms)
                    sweep(std::true_type{});
                else
                    sweep(std::false_type{});
                __syncthreads();  // this CTA's interior updates before anyone's next color
                cluster_wait();
            }
        }
        // finalize own particles (the predict of the next substep re-reads x, v)
        const bool last = s + 1 == substeps;
        if (!last || (flags & kEndFinalize)) {
            for (uint32_t k = tid; k < cnt; k += nthr) {
                const uint32_t i = base + k;
                const float4 p4 = xs[cluster_slot(k)];
                if (p4.w <= 0.0f) continue;
                const V3 xo = v3(W.x[i]);
                V3 vel = v3(W.v[i]);
                const V3 xn = finalize(v3(p4), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, p4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
            }
            pending = false;
        } else {
            for (uint32_t k = tid; k < cnt; k += nthr) W.jac[0][base + k] = xs[cluster_slot(k)];
        }
        __syncthreads();
    }
    // no copy may still target this CTA's shared memory when it exits (every issued chunk was waited for)
    cluster_sync();
}

size_t cluster_gs_smem_bytes(uint32_t shift, uint32_t max_chunk) {
    return ((size_t)16 << shift) + 2 * (size_t)max_chunk * 16 + 2 * sizeof(uint64_t);
}

static const void* cluster_fn(uint32_t cl) {
    if (cl == 8) return (const void*)gs_cluster_kernel<8>;
    if (cl == 16) return (const void*)gs_cluster_kernel<16>;
    return nullptr;
}

bool cluster_gs_supported(uint32_t cl, uint32_t shift, uint32_t max_chunk, uint32_t block) {
    const void* fn = cluster_fn(cl);
    if (!fn) return false;
    const size_t smem = cluster_gs_smem_bytes(shift, max_chunk);
    if (smem > 220 * 1024) return false;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    if (cl > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return false;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return clusters >= 1;
}

cudaError_t launch_cluster_gs(uint32_t cl, uint32_t block, const XpbdWorld& W, const ClusterTable& T,
                              uint32_t flags, uint32_t substeps, uint32_t pend, cudaStream_t st) {
    const void* fn = cluster_fn(cl);
    if (!fn) return cudaErrorInvalidValue;
    const size_t smem = cluster_gs_smem_bytes(T.shift, T.max_chunk);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    XpbdWorld w = W;
    ClusterTable t = T;
    void* args[] = {&w, &t, &flags, &substeps, &pend};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace xpbd
