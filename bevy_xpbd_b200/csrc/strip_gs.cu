// Colored Gauss–Seidel over several thread-block clusters ("strips") for sheets too large to sweep fast on one cluster.
//
// Same arithmetic as the other Gauss–Seidel executions (gs_constraint, xpbd_cpu.rs:349-385; WGSL gs_edges,
// cloth_sim.wgsl:154-210): within a color the constraints are particle-disjoint, so any order inside a color gives
// the reference's sequential result; colors run one after another.
//
// Layout. The packed particles are split into S·CL consecutive ranges, one per CTA; CTAs [s·CL, (s+1)·CL) form
// cluster s (a strip). A particle is "shared" when some constraint joins it to a particle of another strip: shared
// particles live in global memory (one float4 slot each, the authoritative copy for the frame); every other particle
// lives in the shared memory of the CTA that owns it, reached by the strip's other CTAs through distributed shared
// memory. A constraint is solved by the CTA owning its endpoint i. Per (color, CTA) the records come in three kinds:
//   0  touches a shared particle        — global loads/stores, ordered across strips by step flags
//   1  touches a particle another CTA of the strip also touches — distributed shared memory
//   2  touches only particles no other CTA touches — this CTA's shared memory
// Cross-strip order. Each CTA that shares particles with CTAs of other strips ("dependencies", symmetric) counts the
// steps it has completed in a global flag: before touching shared particles in step g it waits until every
// dependency has completed step g - 1 (its flag reaches base + g), and after its kind-0 records it publishes g + 1
// (fence, then a release store). Steps: per substep the predict (which also writes the previous substep's result
// back), then one step per color of every pass; the finalize at the end of the launch waits for the last color.
// Within a strip the colors are separated by the cluster barrier (arrive after the kinds 0 and 1, wait after kind 2).
// Every wait is bounded: after `barrier_timeout_ns` the kernel records XPBD_DEV_BARRIER_TIMEOUT and stops.
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_cluster.h"
#include "xpbd_device.h"
#include "xpbd_fpdiv.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {

namespace {

constexpr uint32_t kSharedBit = 0x80000000u;

__device__ __forceinline__ float4 ld_gpu(const float4* p) {
    float4 v;
    asm volatile("ld.relaxed.gpu.global.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_gpu(float4* p, float4 v) {
    asm volatile("st.relaxed.gpu.global.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z),
                 "f"(v.w)
                 : "memory");
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Endpoint access by code: shared slot (global), or (rank << 16 | local) in the strip's distributed shared memory.
struct Where {
    bool shared;
    uint32_t addr;  // shared-memory address (local window or cluster window)
    float4* g;      // global slot
};
template <int KIND>
__device__ __forceinline__ Where where(uint32_t code, uint32_t xs_base, const uint32_t* s_rank_base,
                                       const StripTable& T) {
    Where w;
    w.shared = KIND == 0 && (code & kSharedBit) != 0u;
    w.g = T.gx + (code & ~kSharedBit);
    const uint32_t local = (code & 0xFFFFu) << 4;
    w.addr = (KIND == 2 ? xs_base : s_rank_base[(code >> 16) & 0x7FFFu]) + local;
    return w;
}
template <int KIND>
__device__ __forceinline__ float4 ld_where(const Where& w) {
    if (KIND == 0 && w.shared) return ld_gpu(w.g);
    return KIND == 2 ? ld_local(w.addr) : ld_dsmem(w.addr);
}
template <int KIND>
__device__ __forceinline__ void st_where(const Where& w, float4 v) {
    if (KIND == 0 && w.shared)
        st_gpu(w.g, v);
    else if (KIND == 2)
        st_local(w.addr, v);
    else
        st_dsmem(w.addr, v);
}

// One constraint of the reference's colored sweep (xpbd_cpu.rs:349-385): both endpoints move by their clamped
// corrections, pinned endpoints stay.
template <int KIND>
__device__ __forceinline__ void strip_solve(const uint4 r, uint32_t xs_base, const uint32_t* s_rank_base,
                                            const StripTable& T, const XpbdDevParams& P) {
    const Where wi = where<KIND>(r.x, xs_base, s_rank_base, T);
    const Where wj = where<KIND>(r.y, xs_base, s_rank_base, T);
    const float4 pi4 = ld_where<KIND>(wi);
    const float4 pj4 = ld_where<KIND>(wj);
    const float w_i = pi4.w, w_j = pj4.w;
    if (w_j <= 0.0f && w_i <= 0.0f) return;
    const F3 p_i = f3(pi4), p_j = f3(pj4);
    F3 gv = sub3(p_i, p_j);
    const float len = len3(gv);
    if (len < 1e-8f) return;
    {
        F3 q;
        if (!fpdiv3_by_length_fast(gv.x, gv.y, gv.z, len, q.x, q.y, q.z)) q = div3(gv, len);
        gv = q;
    }
    const float C = __fsub_rn(len, __uint_as_float(r.z));
    const float alpha_t = __fmul_rn(__uint_as_float(r.w), P.inv_dt_sq);
    const float wsum = __fadd_rn(__fadd_rn(w_i, w_j), alpha_t);
    if (wsum < 1e-8f) return;
    const float dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, 0.0f)), wsum);
    const F3 og = {__fmul_rn(P.omega, gv.x), __fmul_rn(P.omega, gv.y), __fmul_rn(P.omega, gv.z)};
    const F3 dx_i = clamp_correction(mul3(mul3(og, w_i), dlam));
    const F3 dxj = mul3(mul3(og, w_j), dlam);
    const F3 dx_j = clamp_correction(F3{-dxj.x, -dxj.y, -dxj.z});
    if (w_i > 0.0f) {
        const F3 n = add3(p_i, dx_i);
        st_where<KIND>(wi, make_float4(n.x, n.y, n.z, w_i));
    }
    if (w_j > 0.0f) {
        const F3 n = add3(p_j, dx_j);
        st_where<KIND>(wj, make_float4(n.x, n.y, n.z, w_j));
    }
}

}  // namespace

// Record ranges of one (color, CTA) group by kind, and this thread's first record of each kind.
struct Group {
    uint32_t k[4];
    uint4 r[3];
};
__device__ __forceinline__ Group load_group(const StripTable& T, uint32_t c, uint32_t cta, uint32_t tid) {
    Group g;
    const uint32_t* off = T.off + ((size_t)c * T.ncta + cta) * 3;
#pragma unroll
    for (int q = 0; q < 4; ++q) g.k[q] = __ldg(off + q);
#pragma unroll
    for (int q = 0; q < 3; ++q) g.r[q] = g.k[q] + tid < g.k[q + 1] ? __ldg(T.rec + g.k[q] + tid) : make_uint4(0, 0, 0, 0);
    return g;
}

// Waits until every dependency of this CTA has completed step `target` (flag - target >= 0, wrapping); false when
// the bounded wait gave up or another CTA reported an error.
__device__ __forceinline__ bool strip_wait(const XpbdWorld& W, const StripTable& T, uint32_t cta, unsigned target,
                                           unsigned long long timeout_ns) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        int ok = 1;
        for (uint32_t d = T.dep_off[cta]; d < T.dep_off[cta + 1] && ok; ++d) {
            const unsigned* f = T.flags + T.deps[d];
            unsigned long long t0 = 0;
            for (uint32_t spin = 0;; ++spin) {
                if ((int)(ld_acquire_u32(f) - target) >= 0) break;
                if ((spin & 63u) == 63u) {
                    if (t0 == 0) t0 = now_ns();
                    if (*(volatile int*)W.status != 0 || now_ns() - t0 > timeout_ns || spin > (1u << 30)) {
                        atomicOr(W.status, XPBD_DEV_BARRIER_TIMEOUT);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void strip_publish(const StripTable& T, uint32_t cta, unsigned value) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release_u32(T.flags + cta, value);
    }
}

// A frame of `substeps` substeps (x, v in global memory at both ends).
template <int CL>
__global__ void __launch_bounds__(512, 1) gs_strip_kernel(XpbdWorld W, StripTable T, uint32_t substeps) {
    extern __shared__ __align__(16) float4 xs[];
    __shared__ uint32_t s_rank_base[CL];
    const XpbdDevParams P = *W.params;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t rank = cluster_rank();
    const uint32_t cta = blockIdx.x;  // strips are consecutive clusters
    const uint32_t p0 = cta * T.q;
    const uint32_t np = p0 < W.n ? min(T.q, W.n - p0) : 0u;
    const uint32_t xs_base = smem_u32(xs);
    if (tid < CL) s_rank_base[tid] = map_rank(xs_base, tid);
    const bool has_deps = T.dep_off[cta + 1] > T.dep_off[cta];
    const unsigned base = has_deps ? *(volatile unsigned*)(T.flags + cta) : 0u;
    const unsigned long long tmo = P.barrier_timeout_ns;
    const uint32_t ncol = T.ncolors, I = P.iterations;
    unsigned step = 0;
    bool ok = true;
    __syncthreads();
    // write back the result of a substep (x, v) and predict the next one, own particles
    auto predict_step = [&](bool finalize, bool predict) {
        for (uint32_t k = tid; k < np; k += nthr) {
            const uint32_t i = p0 + k;
            const uint32_t slot = T.slot[i];
            const float4 x4 = W.x[i];
            if (x4.w <= 0.0f) {  // pinned: never moves
                if (predict) {
                    if (slot != 0xFFFFFFFFu) st_gpu(T.gx + slot, x4);
                    else xs[k] = x4;
                }
                continue;
            }
            F3 xo = f3(x4);
            F3 vel = f3(W.v[i]);
            if (finalize) {
                const float4 c = slot != 0xFFFFFFFFu ? ld_gpu(T.gx + slot) : xs[k];
                const F3 xn = finalize_particle(f3(c), xo, vel, P, W.status);
                W.x[i] = make_float4(xn.x, xn.y, xn.z, x4.w);
                W.v[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                xo = xn;
            }
            if (predict) {
                const F3 pos = predict_w(W, i, xo, vel, P);
                const float4 p4 = make_float4(pos.x, pos.y, pos.z, x4.w);
                if (slot != 0xFFFFFFFFu)
                    st_gpu(T.gx + slot, p4);
                else
                    xs[k] = p4;
            }
        }
    };
    for (uint32_t s = 0; s < substeps; ++s) {
        if (has_deps) ok = ok && strip_wait(W, T, cta, base + step, tmo);
        if (ok) predict_step(s > 0, true);
        if (has_deps) strip_publish(T, cta, base + step + 1);
        ++step;
        cluster_sync();
        // A thread's first record of each kind is loaded one color ahead (the records repeat every pass).
        Group g = load_group(T, 0, cta, tid);
        for (uint32_t it = 0; it < I; ++it) {
            for (uint32_t c = 0; c < ncol; ++c, ++step) {
                const Group cur = g;
                g = load_group(T, c + 1 < ncol ? c + 1 : 0u, cta, tid);
                if (has_deps) ok = ok && strip_wait(W, T, cta, base + step, tmo);
                if (ok) {
                    if (cur.k[0] + tid < cur.k[1]) strip_solve<0>(cur.r[0], xs_base, s_rank_base, T, P);
                    for (uint32_t k = cur.k[0] + tid + nthr; k < cur.k[1]; k += nthr)
                        strip_solve<0>(T.rec[k], xs_base, s_rank_base, T, P);
                }
                if (has_deps) strip_publish(T, cta, base + step + 1);
                if (ok) {
                    if (cur.k[1] + tid < cur.k[2]) strip_solve<1>(cur.r[1], xs_base, s_rank_base, T, P);
                    for (uint32_t k = cur.k[1] + tid + nthr; k < cur.k[2]; k += nthr)
                        strip_solve<1>(T.rec[k], xs_base, s_rank_base, T, P);
                }
                cluster_arrive();
                if (ok) {
                    if (cur.k[2] + tid < cur.k[3]) strip_solve<2>(cur.r[2], xs_base, s_rank_base, T, P);
                    for (uint32_t k = cur.k[2] + tid + nthr; k < cur.k[3]; k += nthr)
                        strip_solve<2>(T.rec[k], xs_base, s_rank_base, T, P);
                }
                __syncthreads();
                cluster_wait();
            }
        }
    }
    if (has_deps) ok = ok && strip_wait(W, T, cta, base + step, tmo);
    if (ok) predict_step(true, false);
    if (has_deps) strip_publish(T, cta, base + step + 1);
    cluster_sync();  // no CTA leaves while a peer may still address its shared memory
}

size_t strip_gs_smem_bytes(uint32_t q) { return (size_t)q * 16; }

static const void* strip_fn(uint32_t cl) {
    if (cl == 8) return (const void*)&gs_strip_kernel<8>;
    if (cl == 16) return (const void*)&gs_strip_kernel<16>;
    return nullptr;
}

static cudaLaunchConfig_t strip_cfg(uint32_t cl, uint32_t ncta, uint32_t block, size_t smem, cudaStream_t st,
                                    cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ncta, 1, 1);
    cfg.blockDim = dim3(block, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

// True when all `strips` clusters of `cl` CTAs fit on the device at once (every CTA of the launch must be resident:
// the step flags are waited for across clusters).
bool strip_gs_supported(uint32_t cl, uint32_t strips, uint32_t block, uint32_t q) {
    const void* fn = strip_fn(cl);
    if (!fn || block > 512) return false;
    const size_t smem = strip_gs_smem_bytes(q);
    if (smem > 200 * 1024) return false;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    if (cl > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return false;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = strip_cfg(cl, cl * strips, block, smem, nullptr, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (uint32_t)clusters >= strips;
}

cudaError_t launch_strip_gs(uint32_t cl, uint32_t block, const XpbdWorld& W, const StripTable& T, uint32_t substeps,
                            cudaStream_t st) {
    const void* fn = strip_fn(cl);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = strip_cfg(cl, T.ncta, block, strip_gs_smem_bytes(T.q), st, attr);
    XpbdWorld w = W;
    StripTable t = T;
    void* args[] = {&w, &t, &substeps};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace xpbd
