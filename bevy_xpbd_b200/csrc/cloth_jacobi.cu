// Cloth-resident Jacobi for sm_100a: a whole frame of the reference's Jacobi substeps per cloth, the cloth held in
// shared memory, each constraint solved once per pass.
//
// Reference: predict (xpbd_cpu.rs:38-65), jacobi_edges_pass + jacobi_gather_particle (xpbd_cpu.rs:139-226, WGSL
// jacobi_edges / jacobi_gather, cloth_sim_jacobi.wgsl:143-218) with λ cleared before every pass (xpbd_cpu.rs:267),
// post_velocity (xpbd_cpu.rs:393-409).
//
// Layout. A cloth is solved by one CTA, or by a thread-block cluster of up to 8 CTAs whose distributed shared
// memory holds it: rank r owns a contiguous range of the cloth's particles and keeps, per particle, its position
// (float4, w = inverse mass) and its correction sum (float4, w = incidence count). Positions and velocities leave
// shared memory only at substep boundaries (x, v in global memory). The constraint records stream from global memory
// (8 bytes + the compliance per constraint and pass), grouped by (color, rank).
//
// Order of the sums. The reference gathers each particle's corrections in its neighbour-table row, which lists the
// particle's constraints in increasing batch-sorted index (the cursor scatter of mesh_prep.rs:588-635). The batches
// are greedy colors, so a particle meets at most one constraint per color and its row is sorted by color. Solving the
// colors one after another — every constraint of color c solved once, its two terms added to its two endpoints'
// sums, a CTA / cluster barrier between colors — therefore adds each particle's terms in exactly the row's order,
// bit for bit, without atomics and without solving a constraint twice. A constraint's Δλ and |d| are the same from
// either endpoint and n̂ changes sign exactly, so the j endpoint's term is the negated i term (x − t == x + (−t)).
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_cluster.h"
#include "xpbd_device.h"
#include "xpbd_fpdiv.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {

// cl, threads per CTA, particles per rank: the first class whose cl · rank_cap holds a cloth takes it. The single-CTA
// classes fit four, two and one CTA per SM in its 228 KB of shared memory.
const ClothClass kClothClass[kClothClasses] = {
    {1, 256, 1760}, {1, 512, 3520}, {1, 1024, XPBD_CLOTH_RANK_MAX},
    {2, 1024, XPBD_CLOTH_RANK_MAX}, {4, 1024, XPBD_CLOTH_RANK_MAX}, {8, 1024, XPBD_CLOTH_RANK_MAX},
    {16, 1024, 4096}};

size_t cloth_kernel_smem_bytes(uint32_t cap) { return 2 * (size_t)cap * sizeof(float4); }

template <int CL>
__device__ __forceinline__ void cloth_sync() {
    if (CL == 1)
        __syncthreads();
    else
        cluster_sync();
}

// Shared-memory address of endpoint `ep` ((rank << 13) | local) in the array starting at `base` of every CTA.
template <int CL>
__device__ __forceinline__ float4 ld_ep(uint32_t base, uint32_t ep, uint32_t rank) {
    constexpr uint32_t B = cloth_ep_bits(CL);
    const uint32_t a = base + (ep & ((1u << B) - 1u)) * 16u;
    if (CL == 1) return ld_local(a);
    const uint32_t r = ep >> B;
    return r == rank ? ld_local(a) : ld_dsmem(map_rank(a, r));
}
template <int CL>
__device__ __forceinline__ void add_ep(uint32_t base, uint32_t ep, uint32_t rank, float tx, float ty, float tz,
                                       bool negate) {
    constexpr uint32_t B = cloth_ep_bits(CL);
    const uint32_t a = base + (ep & ((1u << B) - 1u)) * 16u;
    const uint32_t r = CL == 1 ? 0u : ep >> B;
    const bool local = CL == 1 || r == rank;
    const uint32_t ra = local ? a : map_rank(a, r);
    float4 s = local ? ld_local(a) : ld_dsmem(ra);
    if (negate) {
        s.x = __fsub_rn(s.x, tx);
        s.y = __fsub_rn(s.y, ty);
        s.z = __fsub_rn(s.z, tz);
    } else {
        s.x = __fadd_rn(s.x, tx);
        s.y = __fadd_rn(s.y, ty);
        s.z = __fadd_rn(s.z, tz);
    }
    if (local)
        st_local(a, s);
    else
        st_dsmem(ra, s);
}

// One constraint of the current color: the reference's Δλ (λ = 0), then (n̂·w_i)·Δλ into i's sum and the negated
// (n̂·w_j)·Δλ into j's. Nothing is added for a pinned endpoint (its row is empty), for |d| < 1e-8 or w sum < 1e-8
// (the reference skips the constraint / has Δλ = 0: its term is zero, which leaves a sum started at +0 unchanged).
template <int CL>
__device__ __forceinline__ void solve_record(uint2 r, float comp, uint32_t pos_base, uint32_t acc_base,
                                             uint32_t rank, float inv_dt_sq) {
    const uint32_t ei = r.x & 0xFFFFu, ej = r.x >> 16;
    const float4 pi = ld_ep<CL>(pos_base, ei, rank);
    const float4 pj = ld_ep<CL>(pos_base, ej, rank);
    const F3 gv = sub3(f3(pi), f3(pj));
    const float len = len3(gv);
    const float alpha_t = __fmul_rn(comp, inv_dt_sq);
    const float wsum = __fadd_rn(__fadd_rn(pi.w, pj.w), alpha_t);
    if (len < 1e-8f || wsum < 1e-8f) return;
    const float C = __fsub_rn(len, __uint_as_float(r.y));
    const float dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, 0.0f)), wsum);
    F3 n;
    if (!fpdiv3_by_length_fast(gv.x, gv.y, gv.z, len, n.x, n.y, n.z)) fpdiv3(gv.x, gv.y, gv.z, len, n.x, n.y, n.z);
    if (pi.w > 0.0f)
        add_ep<CL>(acc_base, ei, rank, __fmul_rn(__fmul_rn(n.x, pi.w), dlam), __fmul_rn(__fmul_rn(n.y, pi.w), dlam),
                   __fmul_rn(__fmul_rn(n.z, pi.w), dlam), false);
    if (pj.w > 0.0f)
        add_ep<CL>(acc_base, ej, rank, __fmul_rn(__fmul_rn(n.x, pj.w), dlam), __fmul_rn(__fmul_rn(n.y, pj.w), dlam),
                   __fmul_rn(__fmul_rn(n.z, pj.w), dlam), true);
}

// A thread's first two records of a color (k and k + BLOCK), loaded ahead of use.
struct Pref {
    uint2 r0, r1;
    float c0, c1;
};
__device__ __forceinline__ Pref pref_load(const ClothSolveTable& T, uint32_t k, uint32_t k1, uint32_t block) {
    Pref p = {make_uint2(0u, 0u), make_uint2(0u, 0u), 0.0f, 0.0f};
    if (k < k1) {
        p.r0 = __ldg(T.rec + k);
        p.c0 = __ldg(T.comp + k);
    }
    if (k + block < k1) {
        p.r1 = __ldg(T.rec + k + block);
        p.c1 = __ldg(T.comp + k + block);
    }
    return p;
}

// A frame (`substeps` substeps) of one cloth per cluster: T.order[blockIdx.x / CL].
template <int CL, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1024 / BLOCK) jacobi_cloth_kernel(XpbdWorld W, ClothSolveTable T,
                                                                         uint32_t substeps) {
    extern __shared__ float4 s_mem[];
    float4* s_pos = s_mem;
    float4* s_acc = s_mem + T.cap;
    const uint32_t tid = threadIdx.x;
    const uint32_t rank = CL > 1 ? cluster_rank() : 0u;
    const XpbdClothDesc D = T.cloths[T.order[blockIdx.x / CL]];
    const XpbdDevParams P = *W.params;
    const uint32_t p0 = rank * D.q;
    const uint32_t np = p0 < D.n ? min(D.q, D.n - p0) : 0u;
    const uint32_t g0 = D.vtx_off + p0;
    const uint32_t pos_base = smem_u32(s_pos), acc_base = smem_u32(s_acc);
    const uint32_t I = P.iterations;
    const uint32_t* seg = T.seg + D.seg_base + rank;
    for (uint32_t p = tid; p < np; p += BLOCK)  // incidence count of the particle's row (degree averaging)
        s_acc[p] = make_float4(0.0f, 0.0f, 0.0f, (float)(W.row_off[g0 + p + 1] - W.row_off[g0 + p]));
    for (uint32_t s = 0; s < substeps; ++s) {
        for (uint32_t p = tid; p < np; p += BLOCK) {  // predict (pinned particles keep their position)
            const uint32_t g = g0 + p;
            const float4 x4 = W.x[g];
            if (x4.w <= 0.0f) {
                s_pos[p] = x4;
                continue;
            }
            F3 vel = f3(W.v[g]);
            const F3 pos = predict_w(W, g, f3(x4), vel, P);
            s_pos[p] = make_float4(pos.x, pos.y, pos.z, x4.w);
        }
        cloth_sync<CL>();
        // The records of a thread's first two rounds of each color are loaded while the previous color is solved
        // (records do not change between passes: after the last color, color 0's are loaded again).
        uint32_t pk0 = __ldg(seg), pk1 = __ldg(seg + 1);
        Pref pf = pref_load(T, pk0 + tid, pk1, BLOCK);
        for (uint32_t it = 0; it < I; ++it) {
            for (uint32_t c = 0; c < D.colors; ++c) {
                const uint32_t k0 = pk0, k1 = pk1;
                const Pref cur = pf;
                const uint32_t cn = c + 1 < D.colors ? c + 1 : 0u;
                pk0 = __ldg(seg + cn * CL);
                pk1 = __ldg(seg + cn * CL + 1);
                pf = pref_load(T, pk0 + tid, pk1, BLOCK);
                if (k0 + tid < k1) solve_record<CL>(cur.r0, cur.c0, pos_base, acc_base, rank, P.inv_dt_sq);
                if (k0 + tid + BLOCK < k1) solve_record<CL>(cur.r1, cur.c1, pos_base, acc_base, rank, P.inv_dt_sq);
                for (uint32_t k = k0 + tid + 2 * BLOCK; k < k1; k += BLOCK)
                    solve_record<CL>(__ldg(T.rec + k), __ldg(T.comp + k), pos_base, acc_base, rank, P.inv_dt_sq);
                cloth_sync<CL>();
            }
            // the pass's update of the owned particles (jacobi_gather_particle's tail), then at the end of the
            // substep the velocity update
            const bool last = it + 1 == I;
            for (uint32_t p = tid; p < np; p += BLOCK) {
                const float4 ps = s_pos[p];
                if (ps.w <= 0.0f) continue;
                const float4 a = s_acc[p];
                F3 delta = {__fmul_rn(P.omega, a.x), __fmul_rn(P.omega, a.y), __fmul_rn(P.omega, a.z)};
                if (P.relaxation == 1u && a.w > 0.0f) delta = div3(delta, a.w);
                delta = clamp_correction(delta);
                F3 xn = add3(f3(ps), delta);
                s_acc[p] = make_float4(0.0f, 0.0f, 0.0f, a.w);
                if (last) {
                    const uint32_t g = g0 + p;
                    F3 vel;
                    xn = finalize_particle(xn, f3(W.x[g]), vel, P, W.status);
                    W.x[g] = make_float4(xn.x, xn.y, xn.z, ps.w);
                    W.v[g] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                } else {
                    s_pos[p] = make_float4(xn.x, xn.y, xn.z, ps.w);
                }
            }
            if (!last) cloth_sync<CL>();
        }
        if (I == 0) {  // no passes: the predicted positions are the substep's result (xpbd_cpu.rs:302-309)
            for (uint32_t p = tid; p < np; p += BLOCK) {
                const float4 ps = s_pos[p];
                if (ps.w <= 0.0f) continue;
                const uint32_t g = g0 + p;
                F3 vel;
                const F3 xn = finalize_particle(f3(ps), f3(W.x[g]), vel, P, W.status);
                W.x[g] = make_float4(xn.x, xn.y, xn.z, ps.w);
                W.v[g] = make_float4(vel.x, vel.y, vel.z, 0.0f);
            }
        }
        // the next substep's predict touches only this CTA's own particles; its barrier precedes any peer read
    }
    if (CL > 1) cluster_sync();  // no CTA leaves while a peer may still address its shared memory
}

template <int CL, int BLOCK>
static const void* cloth_fn() {
    return (const void*)&jacobi_cloth_kernel<CL, BLOCK>;
}
static const void* cloth_fn_of(int cls) {
    switch (cls) {
        case 0: return cloth_fn<1, 256>();
        case 1: return cloth_fn<1, 512>();
        case 2: return cloth_fn<1, 1024>();
        case 3: return cloth_fn<2, 1024>();
        case 4: return cloth_fn<4, 1024>();
        case 5: return cloth_fn<8, 1024>();
        case 6: return cloth_fn<16, 1024>();
        default: return nullptr;
    }
}

bool cloth_class_launchable(int cls) {
    const ClothClass& K = kClothClass[cls];
    if (K.cl <= 8) return true;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(K.cl, 1, 1);
    cfg.blockDim = dim3(K.block, 1, 1);
    cfg.dynamicSmemBytes = cloth_kernel_smem_bytes(K.rank_cap);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, cloth_fn_of(cls), &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return clusters >= 1;
}

cudaError_t cloth_kernel_prepare() {
    for (int c = 0; c < kClothClasses; ++c) {
        const int bytes = (int)cloth_kernel_smem_bytes(kClothClass[c].rank_cap);
        cudaError_t e = cudaFuncSetAttribute(cloth_fn_of(c), cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
        if (kClothClass[c].cl > 8) {
            e = cudaFuncSetAttribute(cloth_fn_of(c), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_cloth_jacobi(int cls, const XpbdWorld& W, const ClothSolveTable& T, uint32_t substeps,
                               cudaStream_t st) {
    if (cls < 0 || cls >= kClothClasses || T.count == 0) return cudaSuccess;
    const ClothClass& K = kClothClass[cls];
    if (T.cap > K.rank_cap) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(T.count * K.cl, 1, 1);
    cfg.blockDim = dim3(K.block, 1, 1);
    cfg.dynamicSmemBytes = cloth_kernel_smem_bytes(T.cap);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K.cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = K.cl > 1 ? 1 : 0;
    XpbdWorld w = W;
    ClothSolveTable t = T;
    void* args[] = {&w, &t, &substeps};
    return cudaLaunchKernelExC(&cfg, cloth_fn_of(cls), args);
}

// ---------------------------------------------------------------------------------------------- one small batch
// Latency path for a single small cloth (or a few): the whole batch spread over one cluster of CL CTAs, thread per
// incidence, one cluster barrier per pass. Rank r owns particles [r·q, (r+1)·q) and their neighbour-table rows; its
// shared memory holds the two Jacobi position buffers of those particles (the reference's jac_a / jac_b ping-pong),
// the rank's constraint records and one correction term per incidence. A pass: every thread evaluates one record —
// the reference's Δλ, times n̂·w of an endpoint (jacobi_edges + jacobi_gather, xpbd_cpu.rs:139-226) — reading the
// other endpoint from its owner's shared memory; a constraint whose endpoints are both on this rank is solved once and
// writes both endpoints' terms, one that joins two ranks is evaluated on each side for its own endpoint; then each
// particle sums its row's terms in table order and writes its new position into the other buffer; a cluster barrier
// ends the pass. Evaluating the cross-rank constraints twice keeps the pass to one barrier: for a small cloth the
// pass is latency-bound.
// The terms sit in shared memory row by row with an odd stride of float4 slots (row p, slot u at p·stride + u): an
// incidence writes its slot, and when the row owners read slot u of their rows, eight consecutive owners (one
// 128-byte phase of a 16-byte load) fall on eight different bank groups. The stride is 4·ceil(longest row / 4) + 1;
// the slots past a row's end are zeroed once and never written, so an owner reads stride − 1 slots without a bound
// test (a +0 term leaves a sum started at +0 unchanged: such a sum never becomes −0). Each row owner computes its
// 1/degree once per launch, so the degree-averaged update needs only the shared-reciprocal steps.
// The particles' x and v stay in shared memory for the whole frame (the predict and the velocity update of every
// substep read and write them there; global memory is read at the start and written at the end).
size_t small_batch_smem_bytes(uint32_t q, uint32_t m_max, uint32_t stride) {
    return 4 * (size_t)q * 16 + (size_t)m_max * 16 + (size_t)q * stride * 16;
}

template <int CL>
__global__ void __launch_bounds__(1024, 1) jacobi_small_batch_kernel(XpbdWorld W, SmallBatch B, uint32_t substeps) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t q = B.q;
    float4* s_pos0 = reinterpret_cast<float4*>(smem);
    float4* s_x = s_pos0 + 2 * (size_t)q;
    float4* s_v = s_x + q;
    uint4* s_rec = reinterpret_cast<uint4*>(smem + 4 * (size_t)q * 16);
    float4* s_term = reinterpret_cast<float4*>(smem + 4 * (size_t)q * 16 + (size_t)B.m_max * 16);
    const uint32_t stride = B.stride;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x;
    const uint32_t rank = cluster_rank();
    const uint32_t p0 = rank * q;
    const uint32_t np = p0 < W.n ? min(q, W.n - p0) : 0u;
    const XpbdDevParams P = *W.params;
    const uint32_t m = B.rbase[rank + 1] - B.rbase[rank];  // records of this rank
    // the launch has at least q threads (small_batch_supported): thread p owns row p for the whole frame, and keeps
    // its degree and its reciprocal in registers
    const uint32_t my_deg = tid < np ? B.roff[rank * (q + 1) + tid + 1] - B.roff[rank * (q + 1) + tid] : 0u;
    const float my_rdeg = my_deg ? __frcp_rn((float)my_deg) : 0.f;
    for (uint32_t k = tid; k < m; k += nthr) s_rec[k] = B.rec[B.rbase[rank] + k];
    for (uint32_t k = tid; k < q * stride; k += nthr) s_term[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    for (uint32_t p = tid; p < np; p += nthr) {
        s_x[p] = W.x[p0 + p];
        s_v[p] = W.v[p0 + p];
    }
    const uint32_t pos_base = smem_u32(s_pos0);
    uint32_t b = 0;  // buffer the next predict writes: never the one a peer may still be reading
    const uint32_t I = P.iterations;
    __syncthreads();
    for (uint32_t s = 0; s < substeps; ++s) {
        for (uint32_t p = tid; p < np; p += nthr) {
            const uint32_t g = p0 + p;
            const float4 x4 = s_x[p];
            float4 out = x4;
            if (x4.w > 0.0f) {
                F3 vel = f3(s_v[p]);
                const F3 pos = predict_w(W, g, f3(x4), vel, P);
                out = make_float4(pos.x, pos.y, pos.z, x4.w);
            }
            if (x4.w > 0.0f)
                s_pos0[b * q + p] = out;
            else if (s == 0)  // pinned: the same in both buffers, for the whole frame
                s_pos0[p] = s_pos0[q + p] = x4;
        }
        cluster_sync();
        for (uint32_t it = 0; it < I; ++it) {
            const uint32_t src = pos_base + b * q * 16u;
            for (uint32_t k = tid; k < m; k += nthr) {
                const uint4 r = s_rec[k];
                const uint32_t self = r.x & 0xFFFFu;  // {slot in the row << 16 | self local}
                const float4 ps = ld_local(src + self * 16u);
                const uint32_t ro = (r.y >> 12) & 0xFu;  // {local | rank << 12 | slot << 16 | both << 31}
                const uint32_t ao = src + (r.y & 0xFFFu) * 16u;
                const float4 po = ro == rank ? ld_local(ao) : ld_dsmem(map_rank(ao, ro));
                const F3 gv = sub3(f3(ps), f3(po));
                const float len = len3(gv);
                const float alpha_t = __fmul_rn(__uint_as_float(r.w), P.inv_dt_sq);
                const float wsum = __fadd_rn(__fadd_rn(ps.w, po.w), alpha_t);
                float4 t = make_float4(0.0f, 0.0f, 0.0f, 0.0f), to = t;
                if (!(len < 1e-8f) && !(wsum < 1e-8f)) {
                    F3 n;
                    if (!fpdiv3_by_length_fast(gv.x, gv.y, gv.z, len, n.x, n.y, n.z))
                        fpdiv3(gv.x, gv.y, gv.z, len, n.x, n.y, n.z);
                    const float C = __fsub_rn(len, __uint_as_float(r.z));
                    const float dlam = __fdiv_rn(__fsub_rn(-C, __fmul_rn(alpha_t, 0.0f)), wsum);
                    t = make_float4(__fmul_rn(__fmul_rn(n.x, ps.w), dlam), __fmul_rn(__fmul_rn(n.y, ps.w), dlam),
                                    __fmul_rn(__fmul_rn(n.z, ps.w), dlam), 0.0f);
                    // the other endpoint's term as its own row evaluates it: the difference, n̂ and so every
                    // product negate exactly, |d|, C, the w sum (two terms commute) and Δλ are the same
                    to = make_float4(__fmul_rn(__fmul_rn(-n.x, po.w), dlam), __fmul_rn(__fmul_rn(-n.y, po.w), dlam),
                                     __fmul_rn(__fmul_rn(-n.z, po.w), dlam), 0.0f);
                }
                s_term[self * stride + (r.x >> 16)] = t;
                if (r.y >> 31) s_term[(r.y & 0xFFFu) * stride + ((r.y >> 16) & 0x7FFFu)] = to;
            }
            __syncthreads();
            const bool last = it + 1 == I;
            const uint32_t p = tid;
            const float4 ps = p < np ? s_pos0[b * q + p] : make_float4(0.f, 0.f, 0.f, 0.f);
            if (ps.w > 0.0f) {  // a free particle of this rank (pinned ones keep their position)
                float ax = 0.0f, ay = 0.0f, az = 0.0f;
                // four terms loaded at once, then added in table order; the slots past the row's end hold +0
                const float4* row = s_term + p * stride;
                for (uint32_t k = 0; k + 1 < stride; k += 4) {
                    float4 t[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) t[u] = row[k + u];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        ax = __fadd_rn(ax, t[u].x);
                        ay = __fadd_rn(ay, t[u].y);
                        az = __fadd_rn(az, t[u].z);
                    }
                }
                F3 delta = {__fmul_rn(P.omega, ax), __fmul_rn(P.omega, ay), __fmul_rn(P.omega, az)};
                if (P.relaxation == 1u && my_deg > 0u)
                    fpdiv3_rcp(delta.x, delta.y, delta.z, (float)my_deg, my_rdeg, delta.x, delta.y, delta.z);
                delta = clamp_correction(delta);
                F3 xn = add3(f3(ps), delta);
                if (last) {
                    F3 vel;
                    xn = finalize_particle(xn, f3(s_x[p]), vel, P, W.status);
                    s_x[p] = make_float4(xn.x, xn.y, xn.z, ps.w);
                    s_v[p] = make_float4(vel.x, vel.y, vel.z, 0.0f);
                }
                s_pos0[(b ^ 1u) * q + p] = make_float4(xn.x, xn.y, xn.z, ps.w);
            }
            b ^= 1u;
            if (!last) cluster_sync();
        }
        if (I == 0) {
            for (uint32_t p = tid; p < np; p += nthr) {
                const float4 ps = s_pos0[b * q + p];
                if (ps.w <= 0.0f) continue;
                F3 vel;
                const F3 xn = finalize_particle(f3(ps), f3(s_x[p]), vel, P, W.status);
                s_x[p] = make_float4(xn.x, xn.y, xn.z, ps.w);
                s_v[p] = make_float4(vel.x, vel.y, vel.z, 0.0f);
            }
        }
        // the last pass read buffer b ^ 1 (peers may still be reading it) and wrote b: the next predict writes b
        __syncthreads();
    }
    for (uint32_t p = tid; p < np; p += nthr) {  // each particle's own thread wrote its x and v
        W.x[p0 + p] = s_x[p];
        W.v[p0 + p] = s_v[p];
    }
    cluster_sync();
}

static const void* small_fn(uint32_t cl) {
    if (cl == 8) return (const void*)&jacobi_small_batch_kernel<8>;
    if (cl == 16) return (const void*)&jacobi_small_batch_kernel<16>;
    return nullptr;
}

static cudaLaunchConfig_t small_cfg(uint32_t cl, uint32_t block, size_t smem, cudaStream_t st,
                                    cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl, 1, 1);
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

bool small_batch_supported(uint32_t cl, uint32_t block, uint32_t q, uint32_t m_max, uint32_t stride) {
    const void* fn = small_fn(cl);
    if (!fn || block > 1024 || q > block) return false;
    const size_t smem = small_batch_smem_bytes(q, m_max, stride);
    if (smem > 220 * 1024) return false;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    if (cl > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return false;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = small_cfg(cl, block, smem, nullptr, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return clusters >= 1;
}

cudaError_t launch_small_batch(uint32_t cl, uint32_t block, const XpbdWorld& W, const SmallBatch& B,
                               uint32_t substeps, cudaStream_t st) {
    const void* fn = small_fn(cl);
    if (!fn) return cudaErrorInvalidValue;
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = small_cfg(cl, block, small_batch_smem_bytes(B.q, B.m_max, B.stride), st, attr);
    XpbdWorld w = W;
    SmallBatch b = B;
    void* args[] = {&w, &b, &substeps};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace xpbd
