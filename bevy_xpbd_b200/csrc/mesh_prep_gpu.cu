// Mesh preparation on the GPU (sm_100a): the greedy edge coloring of partition_constraints_for_gs_batches
// (mesh_prep.rs:153-221) and the particle-major neighbour table of finalize_cloth_mesh (mesh_prep.rs:588-635).
//
// Coloring. The reference colors constraints one at a time in a fixed processing order — (max endpoint degree
// descending, min endpoint, max endpoint, index) (mesh_prep.rs:172-177, a stable sort) — giving each the smallest
// color not yet used at either endpoint (:183-202), then orders the batches by (color, index) (:204-205). The color a
// constraint gets depends only on the colors of the constraints that share a particle with it and come earlier in
// that order. So a Jones–Plassmann schedule whose priority is the processing rank produces the same coloring: a
// constraint is colored once every earlier-ranked neighbour is, in rounds separated by a grid barrier. The number of
// rounds is the longest chain of adjacent constraints with increasing rank — about 10 per vertex of a square sheet's
// side — and the cloths of a batch (disjoint particle ranges, so never adjacent) advance in the same rounds; their
// relative order inside a cloth is unchanged by the cloth's particle offset, so each cloth gets its own coloring.
//
// Steps: degrees (atomics) → processing rank by three stable LSD radix sorts (max endpoint, then min endpoint, then
// degree descending) → particle → constraint adjacency → the rounds: per constraint the number of earlier-ranked
// neighbour slots, then rounds over a frontier (four frontier constraints per warp, 8 lanes each: OR of the
// neighbours' colors in 64-color windows, the smallest free color, release of later-ranked neighbours whose count
// reaches zero) — per cloth in one CTA each when the caller gives the cloths' constraint ranges (jp_cloth_kernel,
// __syncthreads between rounds), else over the whole grid in one cooperative launch (jp_color_kernel, grid barrier
// between rounds) → stable sort by color (the (color, index) batch order) → batch offsets.
//
// Neighbour table. Row p lists the constraints at particle p in increasing constraint position, the i slot of a
// constraint before its j slot — the order of the reference's cursor scatter. That is a stable sort of the 2E
// incidences (2k: particle i of constraint k, 2k+1: particle j) by particle.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <chrono>
#include <vector>
#include <cstdio>
#include <cstdlib>

#include "../../include/xpbd_cuda.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {
namespace {

constexpr unsigned kMask = 0xFFFFFFFFu;
constexpr uint32_t kNoColor = 0xFFFFFFFFu;
constexpr int kPrepBlock = 256;
constexpr int kJpBlock = 1024;
constexpr unsigned long long kPrepBarrierTimeoutNs = 2000000000ull;

// Control words at the start of the scratch.
enum : uint32_t {
    kCtlCount0 = 0,  // frontier sizes, rotating over three words (round r reads word r % 3)
    kCtlStatus = 4,  // XPBD_DEV_* bits
    kCtlRounds = 5,
    kCtlColors = 6,  // largest color + 1
    kCtlDone = 7,    // constraints colored
    kCtlMaxDeg = 8,
    kCtlT0 = 10,     // globaltimer stamps (two words each): kernel start, end of phase 0, end of the rounds
    kCtlT1 = 12,
    kCtlT2 = 14,
    kCtlQueue = 16,    // per-cloth schedule: next entry of the cloth queue
    kCtlBarrier = 32,  // in its own 128-byte line, apart from the frontier counters
    kCtlWords = 64,    // 256 bytes
};
constexpr uint32_t kStatusSchedule = 0x100u;  // a constraint was reached before an earlier-ranked neighbour
constexpr uint32_t kStatusCloth = 0x200u;     // per-cloth schedule: two cloths share a particle

struct ColorLayout {  // offsets in 32-bit words from the scratch base; every array starts on 256 bytes
    size_t ctl, deg, cursor, adj, ka, va, kb, vb, rc, pending, front0, front1, coff, queue, radix;
    size_t radix_bytes, total_bytes;
};

size_t take_words(size_t& off, size_t words) {
    const size_t o = off;
    off += (words + 63) & ~(size_t)63;
    return o;
}

ColorLayout color_layout(uint32_t n, uint32_t e, uint32_t num_cloths) {
    ColorLayout L{};
    size_t off = 0;
    L.ctl = take_words(off, kCtlWords);
    L.deg = take_words(off, (size_t)n + 1);
    L.cursor = take_words(off, n);
    L.adj = take_words(off, 2 * (size_t)e);
    L.ka = take_words(off, e);
    L.va = take_words(off, e);
    L.kb = take_words(off, e);
    L.vb = take_words(off, e);
    L.rc = take_words(off, 2 * (size_t)e);
    L.pending = take_words(off, e);
    L.front0 = take_words(off, e);
    L.front1 = take_words(off, e);
    L.coff = take_words(off, (size_t)num_cloths + 1);
    L.queue = take_words(off, num_cloths);
    L.radix = off;
    L.radix_bytes = radix_sort_scratch_bytes(std::max<uint32_t>(e, 1u));
    L.total_bytes = off * 4 + L.radix_bytes;
    return L;
}

struct TableLayout {
    size_t ctl, keys, vals, skeys, radix;
    size_t radix_bytes, total_bytes;
};

TableLayout table_layout(uint32_t e) {
    TableLayout L{};
    size_t off = 0;
    const size_t m = 2 * (size_t)e;
    L.ctl = take_words(off, kCtlWords);
    L.keys = take_words(off, m);
    L.vals = take_words(off, m);
    L.skeys = take_words(off, m);
    L.radix = off;
    L.radix_bytes = radix_sort_scratch_bytes((uint32_t)std::max<size_t>(m, 1));
    L.total_bytes = off * 4 + L.radix_bytes;
    return L;
}

// 8-bit radix passes that cover the values 0..max_value.
uint32_t passes_for(uint32_t max_value) {
    const uint32_t bits = max_value ? 32u - (uint32_t)__builtin_clz(max_value) : 1u;
    return std::max(1u, (bits + 7u) / 8u);
}

uint32_t grid_for(size_t items, int block) {
    size_t g = (items + block - 1) / block;
    return (uint32_t)std::min<size_t>(std::max<size_t>(g, 1), 148 * 64);
}

// ---------------------------------------------------------------------------------------------- kernels
// Incidence counts per particle; an endpoint out of range (or i == j when reject_self) sets XPBD_DEV_INDEX.
__global__ void degree_kernel(const uint32_t* __restrict__ ci, const uint32_t* __restrict__ cj, uint32_t e,
                              uint32_t n, bool reject_self, uint32_t* __restrict__ deg, uint32_t* __restrict__ ctl) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
        const uint32_t i = ci[k], j = cj[k];
        if (i >= n || j >= n || (reject_self && i == j)) {
            atomicOr(&ctl[kCtlStatus], (unsigned)XPBD_DEV_INDEX);
            continue;
        }
        atomicAdd(&deg[i], 1u);
        atomicAdd(&deg[j], 1u);
    }
}

__global__ void max_degree_kernel(const uint32_t* __restrict__ deg, uint32_t n, uint32_t* __restrict__ ctl) {
    uint32_t m = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, deg[i]);
    m = __reduce_max_sync(kMask, m);
    if ((threadIdx.x & 31u) == 0u && m) atomicMax(&ctl[kCtlMaxDeg], m);
}

// Sort keys of the processing order, one LSD stage each (vals carry the constraint index):
//   stage 0: max endpoint (identity order in), stage 1: min endpoint, stage 2: max_deg - max endpoint degree.
__global__ void order_key_kernel(uint32_t stage, const uint32_t* __restrict__ ci, const uint32_t* __restrict__ cj,
                                 const uint32_t* __restrict__ deg, uint32_t max_deg,
                                 const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
                                 uint32_t* __restrict__ vout, uint32_t e) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
        const uint32_t c = stage == 0 ? k : vin[k];
        const uint32_t i = ci[c], j = cj[c];
        uint32_t key;
        if (stage == 0) key = max(i, j);
        else if (stage == 1) key = min(i, j);
        else key = max_deg - max(deg[i], deg[j]);
        kout[k] = key;
        vout[k] = c;
    }
}

__global__ void adjacency_kernel(const uint32_t* __restrict__ ci, const uint32_t* __restrict__ cj, uint32_t e,
                                 uint32_t* __restrict__ cursor, uint32_t* __restrict__ adj) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
        adj[atomicAdd(&cursor[ci[k]], 1u)] = k;
        adj[atomicAdd(&cursor[cj[k]], 1u)] = k;
    }
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded grid barrier over all blocks of a cooperative launch. One atomic per block on ctl[kCtlBarrier]: block 0
// adds 2^31 - (blocks - 1), the others 1, so the top bit flips when the last block arrives. A wait that exceeds
// kPrepBarrierTimeoutNs (or sees another block's timeout) records XPBD_DEV_BARRIER_TIMEOUT and returns false.
__device__ bool prep_grid_barrier(uint32_t* ctl) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned inc = blockIdx.x == 0 ? (0x80000000u - (gridDim.x - 1u)) : 1u;
        __threadfence();
        const unsigned old = atomicAdd(&ctl[kCtlBarrier], inc);
        unsigned spins = 0;
        unsigned long long t0 = 0;
        while (((old ^ ld_acquire_gpu(&ctl[kCtlBarrier])) & 0x80000000u) == 0u) {
            if ((++spins & 255u) == 0u) {
                if (t0 == 0) t0 = globaltimer_ns();
                if (*(volatile uint32_t*)&ctl[kCtlStatus] & XPBD_DEV_BARRIER_TIMEOUT) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > kPrepBarrierTimeoutNs || spins > (1u << 30)) {
                    atomicOr(&ctl[kCtlStatus], (unsigned)XPBD_DEV_BARRIER_TIMEOUT);
                    ok = 0;
                    break;
                }
                if (spins > (1u << 16)) __nanosleep(128);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct JpArgs {
    const uint32_t* ci;
    const uint32_t* cj;
    const uint32_t* row_off;  // n + 1
    const uint32_t* adj;      // 2e constraint ids, row p = constraints at particle p
    uint2* rc;                // per constraint {processing rank, color}; colors are written during the rounds
    uint32_t* pending;        // earlier-ranked neighbour slots not yet colored
    uint32_t* front0;
    uint32_t* front1;
    uint32_t* ctl;
    uint32_t e;
};

constexpr uint32_t kGroup = 8;       // lanes per frontier constraint (4 constraints per warp)
constexpr uint32_t kGroupSlots = 4;  // neighbour slots per lane kept in registers (degree sums up to 32)
constexpr uint32_t kPerWarp = 32u / kGroup;

// Neighbour slot t of constraint k: row of its i endpoint first, then row of its j endpoint.
__device__ __forceinline__ uint32_t slot_at(const JpArgs& a, uint32_t t, uint32_t b0, uint32_t l0, uint32_t b1) {
    return __ldg(&a.adj[t < l0 ? b0 + t : b1 + (t - l0)]);
}

// OR over the kGroup lanes of each group; every lane of the warp takes part.
__device__ __forceinline__ unsigned long long group_or(unsigned long long m) {
#pragma unroll
    for (uint32_t o = 1; o < kGroup; o <<= 1) {
        const uint32_t lo = __shfl_xor_sync(kMask, (uint32_t)m, o);
        const uint32_t hi = __shfl_xor_sync(kMask, (uint32_t)(m >> 32), o);
        m |= ((unsigned long long)hi << 32) | lo;
    }
    return m;
}

__device__ __forceinline__ void stamp(uint32_t* ctl, uint32_t word) {
    const unsigned long long t = globaltimer_ns();
    ctl[word] = (uint32_t)t;
    ctl[word + 1] = (uint32_t)(t >> 32);
}

// Loads and stores of the state that changes during a launch (frontiers, colors): across the CTAs of a grid they go
// to L2 (ld.cg / st.cg: another SM's L1 may hold a stale line); inside one CTA, __syncthreads orders them and the
// SM's own L1 is coherent for its threads, so plain accesses serve.
template <bool GRID, typename T>
__device__ __forceinline__ T ld_shared_state(const T* p) {
    if constexpr (GRID) return __ldcg(p);
    else return *p;
}
template <bool GRID>
__device__ __forceinline__ void st_shared_state(uint32_t* p, uint32_t v) {
    if constexpr (GRID) __stcg(p, v);
    else *p = v;
}

// One step of a round for one warp: colors the frontier entries first .. first + 3 of `cur` (one per 8-lane group;
// entries at or beyond `size` are idle) and appends the later-ranked neighbours that become ready to `nxt`, counting
// them in *ncount (global or shared memory). Warp-collective: every lane calls it with the same first and size.
template <bool GRID>
__device__ __forceinline__ void jp_color_group(const JpArgs& a, const uint32_t* cur, uint32_t first, uint32_t size,
                                               uint32_t* nxt, uint32_t* ncount, uint32_t lane, uint32_t& max_color) {
    const uint32_t sub = lane & (kGroup - 1u);
    const uint32_t item = first + lane / kGroup;
    const bool valid = item < size;
    uint32_t k = 0, r = 0, b0 = 0, l0 = 0, b1 = 0, len = 0;
    if (valid) {
        k = ld_shared_state<GRID>(&cur[item]);
        r = ld_shared_state<GRID>(&a.rc[k].x);
        const uint32_t p0 = __ldg(&a.ci[k]), p1 = __ldg(&a.cj[k]);
        b0 = __ldg(&a.row_off[p0]);
        l0 = __ldg(&a.row_off[p0 + 1]) - b0;
        b1 = __ldg(&a.row_off[p1]);
        len = l0 + (__ldg(&a.row_off[p1 + 1]) - b1);
    }
    // colors of the earlier-ranked neighbours, first 64-color window
    uint32_t fs[kGroupSlots], rs[kGroupSlots];
    unsigned long long m = 0;
    bool missing = false;
#pragma unroll
    for (uint32_t j = 0; j < kGroupSlots; ++j) {
        const uint32_t t = sub + kGroup * j;
        fs[j] = kNoColor;
        rs[j] = 0;
        if (t < len) {
            const uint32_t f = slot_at(a, t, b0, l0, b1);
            const uint2 v = ld_shared_state<GRID>(&a.rc[f]);
            fs[j] = f;
            rs[j] = v.x;
            if (f != k && v.x < r) {
                if (v.y == kNoColor) missing = true;
                else if (v.y < 64u) m |= 1ull << v.y;
            }
        }
    }
    for (uint32_t t = sub + kGroup * kGroupSlots; t < len; t += kGroup) {
        const uint32_t f = slot_at(a, t, b0, l0, b1);
        const uint2 v = ld_shared_state<GRID>(&a.rc[f]);
        if (f != k && v.x < r) {
            if (v.y == kNoColor) missing = true;
            else if (v.y < 64u) m |= 1ull << v.y;
        }
    }
    m = group_or(m);
    bool need = valid && m == ~0ull;
    uint32_t col = (valid && !need) ? (uint32_t)__ffsll((long long)~m) - 1u : 0u;
    for (uint32_t base = 64u; __any_sync(kMask, need); base += 64u) {  // rare: 64 colors taken
        unsigned long long w = 0;
        if (need) {
            for (uint32_t t = sub; t < len; t += kGroup) {
                const uint32_t f = slot_at(a, t, b0, l0, b1);
                const uint2 v = ld_shared_state<GRID>(&a.rc[f]);
                if (f != k && v.x < r && v.y != kNoColor && v.y - base < 64u) w |= 1ull << (v.y - base);
            }
        }
        w = group_or(w);
        if (need && w != ~0ull) {
            col = base + (uint32_t)__ffsll((long long)~w) - 1u;
            need = false;
        }
    }
    if (missing) atomicOr(&a.ctl[kCtlStatus], kStatusSchedule);
    if (valid && sub == 0) {
        st_shared_state<GRID>(&a.rc[k].y, col);
        max_color = max(max_color, col + 1u);
    }
    // release the later-ranked neighbours; the ones that become ready join the next frontier with one
    // counter atomic per warp and slot
#pragma unroll
    for (uint32_t j = 0; j < kGroupSlots; ++j) {
        const uint32_t f = fs[j];
        const bool push = valid && f != kNoColor && f != k && rs[j] > r && atomicSub(&a.pending[f], 1u) == 1u;
        const unsigned ballot = __ballot_sync(kMask, push);
        if (ballot) {
            const uint32_t leader = (uint32_t)__ffs(ballot) - 1u;
            uint32_t at = 0;
            if (lane == leader) at = atomicAdd(ncount, (uint32_t)__popc(ballot));
            at = __shfl_sync(kMask, at, leader);
            if (push) st_shared_state<GRID>(&nxt[at + (uint32_t)__popc(ballot & ((1u << lane) - 1u))], f);
        }
    }
    if (!valid) return;
    for (uint32_t t = sub + kGroup * kGroupSlots; t < len; t += kGroup) {
        const uint32_t f = slot_at(a, t, b0, l0, b1);
        if (f != k && ld_shared_state<GRID>(&a.rc[f].x) > r && atomicSub(&a.pending[f], 1u) == 1u)
            st_shared_state<GRID>(&nxt[atomicAdd(ncount, 1u)], f);
    }
}

__global__ void __launch_bounds__(kJpBlock) jp_color_kernel(JpArgs a) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthr = gridDim.x * blockDim.x;
    if (tid == 0) stamp(a.ctl, kCtlT0);
    // phase 0: pending counts and the first frontier (nothing writes rc in this phase)
    for (uint32_t k = tid; k < a.e; k += nthr) {
        const uint32_t r = a.rc[k].x;
        const uint32_t p0 = __ldg(&a.ci[k]), p1 = __ldg(&a.cj[k]);
        uint32_t cnt = 0;
        for (uint32_t q = __ldg(&a.row_off[p0]), q1 = __ldg(&a.row_off[p0 + 1]); q < q1; ++q) {
            const uint32_t f = __ldg(&a.adj[q]);
            cnt += (f != k && a.rc[f].x < r) ? 1u : 0u;
        }
        for (uint32_t q = __ldg(&a.row_off[p1]), q1 = __ldg(&a.row_off[p1 + 1]); q < q1; ++q) {
            const uint32_t f = __ldg(&a.adj[q]);
            cnt += (f != k && a.rc[f].x < r) ? 1u : 0u;
        }
        a.pending[k] = cnt;
        if (cnt == 0) a.front0[atomicAdd(&a.ctl[kCtlCount0], 1u)] = k;
    }
    if (!prep_grid_barrier(a.ctl)) return;
    if (tid == 0) stamp(a.ctl, kCtlT1);
    const uint32_t lane = threadIdx.x & 31u, gw = tid >> 5, nw = nthr >> 5;
    uint32_t max_color = 0;  // largest color + 1 this thread wrote
    for (uint32_t round = 0;; ++round) {
        const uint32_t size = __ldcg(&a.ctl[kCtlCount0 + round % 3]);
        if (size == 0) break;
        if (round > a.e) {  // every round colors at least one constraint, so this never triggers; bounds the loop
            if (tid == 0) atomicOr(&a.ctl[kCtlStatus], kStatusSchedule);
            break;
        }
        if (tid == 0) {
            // word (round + 2) % 3 held the size of round - 1, read by every block before the last barrier; it
            // becomes the counter of round + 2, first incremented after the next barrier
            a.ctl[kCtlCount0 + (round + 2) % 3] = 0;
            a.ctl[kCtlRounds] = round + 1;
            a.ctl[kCtlDone] += size;
        }
        const uint32_t* cur = (round & 1u) ? a.front1 : a.front0;
        uint32_t* nxt = (round & 1u) ? a.front0 : a.front1;
        uint32_t* ncount = &a.ctl[kCtlCount0 + (round + 1) % 3];
        for (uint32_t first = gw * kPerWarp; first < size; first += nw * kPerWarp)  // warp-uniform loop
            jp_color_group<true>(a, cur, first, size, nxt, ncount, lane, max_color);
        if (!prep_grid_barrier(a.ctl)) return;
    }
    max_color = __reduce_max_sync(kMask, max_color);
    if (lane == 0 && max_color) atomicMax(&a.ctl[kCtlColors], max_color);
    if (tid == 0) stamp(a.ctl, kCtlT2);
}

// Per-cloth schedule, for batches whose cloths (contiguous constraint ranges) share no particle: one CTA colors one
// cloth at a time, taking cloths from a queue (largest first), with the frontier counters in shared memory and
// __syncthreads between rounds instead of a grid barrier — a round costs the CTA's own dependent accesses only, and
// no CTA ever waits for another.
__global__ void __launch_bounds__(kJpBlock) jp_cloth_kernel(JpArgs a, const uint32_t* __restrict__ coff,
                                                             const uint32_t* __restrict__ queue,
                                                             uint32_t num_cloths) {
    __shared__ uint32_t s_cnt[3];
    __shared__ uint32_t s_cloth;
    const uint32_t tid = threadIdx.x, nthr = blockDim.x, lane = tid & 31u, wid = tid >> 5, nw = nthr >> 5;
    if (blockIdx.x == 0 && tid == 0) {
        stamp(a.ctl, kCtlT0);
        stamp(a.ctl, kCtlT1);
    }
    uint32_t max_color = 0;
    for (;;) {
        if (tid == 0) s_cloth = atomicAdd(&a.ctl[kCtlQueue], 1u);
        if (tid < 3) s_cnt[tid] = 0;
        __syncthreads();
        const uint32_t qi = s_cloth;
        if (qi >= num_cloths) break;
        const uint32_t cl = queue[qi], c0 = coff[cl], c1 = coff[cl + 1];
        uint32_t* f0 = a.front0 + c0;
        uint32_t* f1 = a.front1 + c0;
        // pending counts and the first frontier; every neighbour must belong to this cloth
        bool foreign = false;
        for (uint32_t k = c0 + tid; k < c1; k += nthr) {
            const uint32_t r = a.rc[k].x;
            const uint32_t p0 = __ldg(&a.ci[k]), p1 = __ldg(&a.cj[k]);
            uint32_t cnt = 0;
            for (uint32_t q = __ldg(&a.row_off[p0]), q1 = __ldg(&a.row_off[p0 + 1]); q < q1; ++q) {
                const uint32_t f = __ldg(&a.adj[q]);
                foreign |= f < c0 || f >= c1;
                cnt += (f != k && a.rc[f].x < r) ? 1u : 0u;
            }
            for (uint32_t q = __ldg(&a.row_off[p1]), q1 = __ldg(&a.row_off[p1 + 1]); q < q1; ++q) {
                const uint32_t f = __ldg(&a.adj[q]);
                foreign |= f < c0 || f >= c1;
                cnt += (f != k && a.rc[f].x < r) ? 1u : 0u;
            }
            a.pending[k] = cnt;
            if (cnt == 0) f0[atomicAdd(&s_cnt[0], 1u)] = k;
        }
        // a cloth sharing a particle with another is not colored (its rounds could release the other cloth's
        // constraints into this cloth's frontier range); adjacency is symmetric, so the other cloth stops too
        if (__syncthreads_or(foreign)) {
            if (tid == 0) atomicOr(&a.ctl[kCtlStatus], kStatusCloth);
            continue;
        }
        uint32_t round = 0;
        for (;; ++round) {
            const uint32_t size = s_cnt[round % 3];
            if (size == 0) break;
            if (round > c1 - c0) {  // every round colors at least one constraint: never taken; bounds the loop
                if (tid == 0) atomicOr(&a.ctl[kCtlStatus], kStatusSchedule);
                break;
            }
            // word (round + 2) % 3 held the size of round - 1, read before the last __syncthreads; it counts the
            // frontier of round + 2, first incremented in round + 1
            if (tid == 0) {
                s_cnt[(round + 2) % 3] = 0;
                atomicAdd(&a.ctl[kCtlDone], size);
            }
            const uint32_t* cur = (round & 1u) ? f1 : f0;
            uint32_t* nxt = (round & 1u) ? f0 : f1;
            for (uint32_t first = wid * kPerWarp; first < size; first += nw * kPerWarp)  // warp-uniform loop
                jp_color_group<false>(a, cur, first, size, nxt, &s_cnt[(round + 1) % 3], lane, max_color);
            __syncthreads();
        }
        if (tid == 0) atomicMax(&a.ctl[kCtlRounds], round);
        __syncthreads();  // s_cnt and s_cloth are rewritten for the next cloth
    }
    max_color = __reduce_max_sync(kMask, max_color);
    if (lane == 0 && max_color) atomicMax(&a.ctl[kCtlColors], max_color);
    if (tid == 0) atomicMax(reinterpret_cast<unsigned long long*>(&a.ctl[kCtlT2]), globaltimer_ns());
}

// rc[k] = {rank, no color}: rank[order[k]] = k (order == nullptr: index order).
__global__ void rank_kernel(const uint32_t* __restrict__ order, uint32_t e, uint2* __restrict__ rc) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x)
        rc[order ? order[k] : k] = make_uint2(k, kNoColor);
}

__global__ void color_extract_kernel(const uint2* __restrict__ rc, uint32_t e, uint32_t* __restrict__ color,
                                     uint32_t* __restrict__ iota) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < e; k += gridDim.x * blockDim.x) {
        color[k] = rc[k].y;
        iota[k] = k;
    }
}

// offsets[c] = first position of color c in the color-sorted order (greedy leaves no color unused); offsets[nc] = e.
__global__ void batch_offsets_kernel(const uint32_t* __restrict__ sorted_colors, uint32_t e, uint32_t ncolors,
                                     uint32_t* __restrict__ offsets) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t k = tid; k < e; k += gridDim.x * blockDim.x) {
        const uint32_t c = sorted_colors[k];
        if (k == 0 || sorted_colors[k - 1] != c) offsets[c] = k;
    }
    if (tid == 0) offsets[ncolors] = e;
}

__global__ void incidence_keys_kernel(const uint32_t* __restrict__ ci, const uint32_t* __restrict__ cj, uint32_t e,
                                      uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t m = 2 * e;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const uint32_t k = q >> 1;
        keys[q] = (q & 1u) ? cj[k] : ci[k];
        vals[q] = q;
    }
}

// eid[p] holds the sorted incidence id q on entry; writes other[p] (the opposite endpoint) and eid[p] = q / 2.
__global__ void incidence_rows_kernel(const uint32_t* __restrict__ ci, const uint32_t* __restrict__ cj, uint32_t e,
                                      uint32_t* __restrict__ other, uint32_t* __restrict__ eid) {
    const uint32_t m = 2 * e;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < m; p += gridDim.x * blockDim.x) {
        const uint32_t q = eid[p], k = q >> 1;
        other[p] = (q & 1u) ? ci[k] : cj[k];
        eid[p] = k;
    }
}

cudaError_t read_ctl(const uint32_t* ctl, uint32_t* host, cudaStream_t st) {
    cudaError_t err = cudaMemcpyAsync(host, ctl, kCtlWords * sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (err != cudaSuccess) return err;
    return cudaStreamSynchronize(st);
}

// XPBD_TRACE=1 in the environment: the device coloring synchronises after each phase and prints its host time
// (and the rounds kernel's own phase times) to stderr. Off, it adds nothing.
struct PrepTrace {
    bool on;
    cudaStream_t st;
    std::chrono::steady_clock::time_point t;
    explicit PrepTrace(cudaStream_t s) : st(s), t(std::chrono::steady_clock::now()) {
        const char* v = getenv("XPBD_TRACE");
        on = v && *v && *v != '0';
    }
    void mark(const char* phase) {
        if (!on) return;
        cudaStreamSynchronize(st);
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "[xpbd] device coloring  %-28s %8.2f ms\n", phase,
                std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

int status_to_error(uint32_t status) {
    if (status & XPBD_DEV_INDEX) return XPBD_ERR_INDEX_RANGE;
    if (status & XPBD_DEV_BARRIER_TIMEOUT) return XPBD_ERR_BARRIER_TIMEOUT;
    if (status & kStatusCloth) return XPBD_ERR_INVALID_ARGUMENT;
    return status ? XPBD_ERR_STATE : XPBD_OK;
}

}  // namespace
}  // namespace xpbd

using namespace xpbd;

extern "C" size_t xpbd_color_constraints_device_scratch_bytes(uint32_t num_particles, uint32_t num_constraints,
                                                              uint32_t num_cloths) {
    return color_layout(num_particles, num_constraints, num_cloths).total_bytes;
}

extern "C" int xpbd_color_constraints_device(uint32_t n, uint32_t e, const uint32_t* ci, const uint32_t* cj,
                                             uint32_t order, uint32_t num_cloths,
                                             const uint32_t* cloth_constraint_offsets, uint32_t* perm,
                                             uint32_t* colors, uint32_t* offsets, uint32_t* batch_count,
                                             void* scratch, size_t scratch_bytes, void* stream) {
    if (!batch_count || !offsets || (e && (!ci || !cj || !perm))) return XPBD_ERR_INVALID_ARGUMENT;
    if (order != XPBD_ORDER_COLOR_REFERENCE && order != XPBD_ORDER_COLOR_INDEX) return XPBD_ERR_INVALID_ARGUMENT;
    if (e > 0x7FFFFFFFu) return XPBD_ERR_CAPACITY;
    if (num_cloths) {  // cloth ranges: contiguous, covering every constraint
        const uint32_t* co = cloth_constraint_offsets;
        if (!co || co[0] != 0 || co[num_cloths] != e) return XPBD_ERR_INVALID_ARGUMENT;
        for (uint32_t k = 0; k < num_cloths; ++k)
            if (co[k + 1] < co[k]) return XPBD_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (e == 0) {  // one empty batch, as the host coloring
        const uint32_t zero[2] = {0, 0};
        if (cudaMemcpyAsync(offsets, zero, sizeof(zero), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return XPBD_ERR_CUDA;
        *batch_count = 1;
        return XPBD_OK;
    }
    const ColorLayout L = color_layout(n, e, num_cloths);
    if (!scratch || scratch_bytes < L.total_bytes || ((uintptr_t)scratch & 255u)) return XPBD_ERR_INVALID_ARGUMENT;
    uint32_t* base = (uint32_t*)scratch;
    uint32_t* ctl = base + L.ctl;
    uint32_t* deg = base + L.deg;
    uint32_t *ka = base + L.ka, *va = base + L.va, *kb = base + L.kb, *vb = base + L.vb;
    uint2* rc = reinterpret_cast<uint2*>(base + L.rc);
    void* radix = base + L.radix;
    PrepTrace trace(st);
    uint32_t h[kCtlWords];
    cudaError_t err = cudaSuccess;
#define PREP_CK(x)                                     \
    do {                                               \
        err = (x);                                     \
        if (err != cudaSuccess) return XPBD_ERR_CUDA;  \
    } while (0)
    PREP_CK(cudaMemsetAsync(ctl, 0, kCtlWords * sizeof(uint32_t), st));
    PREP_CK(cudaMemsetAsync(deg, 0, ((size_t)n + 1) * sizeof(uint32_t), st));
    degree_kernel<<<grid_for(e, kPrepBlock), kPrepBlock, 0, st>>>(ci, cj, e, n, true, deg, ctl);
    max_degree_kernel<<<grid_for(n, kPrepBlock), kPrepBlock, 0, st>>>(deg, n, ctl);
    PREP_CK(cudaGetLastError());
    PREP_CK(read_ctl(ctl, h, st));
    if (h[kCtlStatus]) return status_to_error(h[kCtlStatus]);
    trace.mark("degrees");
    // ---- processing rank
    const uint32_t ge = grid_for(e, kPrepBlock);
    if (order == XPBD_ORDER_COLOR_REFERENCE) {
        const uint32_t pn = passes_for(n - 1);
        order_key_kernel<<<ge, kPrepBlock, 0, st>>>(0, ci, cj, deg, 0, nullptr, ka, va, e);
        PREP_CK(radix_sort_pairs(ka, va, kb, vb, e, pn, radix, L.radix_bytes, st, nullptr));
        order_key_kernel<<<ge, kPrepBlock, 0, st>>>(1, ci, cj, deg, 0, vb, ka, va, e);
        PREP_CK(radix_sort_pairs(ka, va, kb, vb, e, pn, radix, L.radix_bytes, st, nullptr));
        order_key_kernel<<<ge, kPrepBlock, 0, st>>>(2, ci, cj, deg, h[kCtlMaxDeg], vb, ka, va, e);
        PREP_CK(radix_sort_pairs(ka, va, kb, vb, e, passes_for(h[kCtlMaxDeg]), radix, L.radix_bytes, st, nullptr));
        rank_kernel<<<ge, kPrepBlock, 0, st>>>(vb, e, rc);
    } else {
        rank_kernel<<<ge, kPrepBlock, 0, st>>>(nullptr, e, rc);
    }
    trace.mark("processing rank (3 sorts)");
    // ---- particle → constraint adjacency (row order is irrelevant to the coloring)
    PREP_CK(launch_exclusive_scan(deg, n + 1, nullptr, st));
    PREP_CK(cudaMemcpyAsync(base + L.cursor, deg, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    adjacency_kernel<<<ge, kPrepBlock, 0, st>>>(ci, cj, e, base + L.cursor, base + L.adj);
    PREP_CK(cudaGetLastError());
    trace.mark("adjacency");
    // ---- Jones–Plassmann rounds: per cloth (one CTA each, largest first) when the caller gives the cloth ranges,
    // else over the whole grid (one cooperative launch, grid barrier per round)
    int dev = 0, sms = 0, per_sm = 0;
    PREP_CK(cudaGetDevice(&dev));
    PREP_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    JpArgs a{ci, cj, deg, base + L.adj, rc, base + L.pending, base + L.front0, base + L.front1, ctl, e};
    uint32_t blocks = 0;
    if (num_cloths) {
        std::vector<uint32_t> queue(num_cloths);
        for (uint32_t k = 0; k < num_cloths; ++k) queue[k] = k;
        const uint32_t* co = cloth_constraint_offsets;
        std::stable_sort(queue.begin(), queue.end(),
                         [&](uint32_t x, uint32_t y) { return co[x + 1] - co[x] > co[y + 1] - co[y]; });
        PREP_CK(cudaMemcpyAsync(base + L.coff, co, ((size_t)num_cloths + 1) * 4, cudaMemcpyHostToDevice, st));
        PREP_CK(cudaMemcpyAsync(base + L.queue, queue.data(), (size_t)num_cloths * 4, cudaMemcpyHostToDevice, st));
        PREP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jp_cloth_kernel, kJpBlock, 0));
        if (per_sm < 1) return XPBD_ERR_UNSUPPORTED;
        blocks = std::min<uint32_t>(num_cloths, (uint32_t)(sms * per_sm));
        jp_cloth_kernel<<<blocks, kJpBlock, 0, st>>>(a, base + L.coff, base + L.queue, num_cloths);
        PREP_CK(cudaGetLastError());
        PREP_CK(cudaStreamSynchronize(st));  // the host queue array must outlive its copy
    } else {
        PREP_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jp_color_kernel, kJpBlock, 0));
        if (per_sm < 1) return XPBD_ERR_UNSUPPORTED;
        blocks = (uint32_t)(sms * per_sm);
        void* args[] = {&a};
        PREP_CK(cudaLaunchCooperativeKernel((const void*)jp_color_kernel, dim3(blocks), dim3(kJpBlock), args, 0, st));
    }
    PREP_CK(read_ctl(ctl, h, st));
    if (h[kCtlStatus]) return status_to_error(h[kCtlStatus]);
    if (h[kCtlDone] != e) return XPBD_ERR_INDEX_RANGE;
    const uint32_t ncolors = h[kCtlColors];
    if (trace.on) {
        auto span = [&](uint32_t w0, uint32_t w1) {
            const uint64_t t0 = h[w0] | ((uint64_t)h[w0 + 1] << 32), t1 = h[w1] | ((uint64_t)h[w1 + 1] << 32);
            return (double)(t1 - t0) * 1e-6;
        };
        fprintf(stderr, "[xpbd] device coloring  pending counts %8.2f ms, %u rounds %8.2f ms (%u blocks x %d)\n",
                span(kCtlT0, kCtlT1), h[kCtlRounds], span(kCtlT1, kCtlT2), blocks, kJpBlock);
    }
    trace.mark("rounds (one launch)");
    // ---- (color, index) batch order and offsets
    color_extract_kernel<<<ge, kPrepBlock, 0, st>>>(rc, e, ka, va);
    PREP_CK(radix_sort_pairs(ka, va, kb, perm, e, passes_for(ncolors - 1), radix, L.radix_bytes, st, nullptr));
    batch_offsets_kernel<<<ge, kPrepBlock, 0, st>>>(kb, e, ncolors, offsets);
    if (colors) PREP_CK(cudaMemcpyAsync(colors, ka, (size_t)e * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    PREP_CK(cudaGetLastError());
    trace.mark("batch order");
    *batch_count = ncolors;
    return XPBD_OK;
#undef PREP_CK
}

extern "C" size_t xpbd_neighbor_table_device_scratch_bytes(uint32_t num_particles, uint32_t num_constraints) {
    (void)num_particles;
    return table_layout(num_constraints).total_bytes;
}

extern "C" int xpbd_neighbor_table_device(uint32_t n, uint32_t e, const uint32_t* ci, const uint32_t* cj,
                                          uint32_t* row_off, uint32_t* other, uint32_t* eid, void* scratch,
                                          size_t scratch_bytes, void* stream) {
    if (!row_off || (e && (!ci || !cj || !other || !eid))) return XPBD_ERR_INVALID_ARGUMENT;
    if (e > 0x7FFFFFFFu) return XPBD_ERR_CAPACITY;
    const TableLayout L = table_layout(e);
    if (!scratch || scratch_bytes < L.total_bytes || ((uintptr_t)scratch & 255u)) return XPBD_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* base = (uint32_t*)scratch;
    uint32_t* ctl = base + L.ctl;
    uint32_t h[kCtlWords];
    const uint32_t m = 2 * e;
    if (cudaMemsetAsync(ctl, 0, kCtlWords * sizeof(uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(row_off, 0, ((size_t)n + 1) * sizeof(uint32_t), st) != cudaSuccess)
        return XPBD_ERR_CUDA;
    if (e) degree_kernel<<<grid_for(e, kPrepBlock), kPrepBlock, 0, st>>>(ci, cj, e, n, false, row_off, ctl);
    if (cudaGetLastError() != cudaSuccess || read_ctl(ctl, h, st) != cudaSuccess) return XPBD_ERR_CUDA;
    if (h[kCtlStatus]) return status_to_error(h[kCtlStatus]);
    if (launch_exclusive_scan(row_off, n + 1, nullptr, st) != cudaSuccess) return XPBD_ERR_CUDA;
    if (e) {
        const uint32_t g = grid_for(m, kPrepBlock);
        incidence_keys_kernel<<<g, kPrepBlock, 0, st>>>(ci, cj, e, base + L.keys, base + L.vals);
        if (radix_sort_pairs(base + L.keys, base + L.vals, base + L.skeys, eid, m, passes_for(n ? n - 1 : 0),
                             base + L.radix, L.radix_bytes, st, nullptr) != cudaSuccess)
            return XPBD_ERR_CUDA;
        incidence_rows_kernel<<<g, kPrepBlock, 0, st>>>(ci, cj, e, other, eid);
    }
    return cudaGetLastError() == cudaSuccess ? XPBD_OK : XPBD_ERR_CUDA;
}
