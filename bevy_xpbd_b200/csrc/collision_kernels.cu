// Self-collision for sm_100a: spatial-hash keys, stable LSD radix sort of (32-bit key, particle) pairs, bucket
// table, 27-cell neighbour query with the reference narrow phase.
//
// Reference: the GPU path of cloth_sim_jacobi.wgsl (keys :243-253, radix sort :299-355, cell ranges :362-384,
// collide_grid_cells + narrow_self_collision_pair :386-470, collide_apply :472-490) and the CPU solver it is judged
// against, self_collision_resolve (xpbd_cpu.rs:67-137). Differences by design:
//   * keys: integer cell coordinates floor(x / cell) hashed with the primes 73856093 / 19349663 / 83492791 (XOR of
//     wrapping u32 products) into a 2^bits table, instead of a dense clamped grid;
//   * the sort is stable (per-tile ranks from warp match_any in input order) — the reference's atomic scatter is not;
//   * accumulation is deterministic: each particle gathers its own partners and sums their corrections in increasing
//     partner index, which is exactly the order of the reference's all-pairs loop, so the FP32 result matches
//     self_collision_resolve bit for bit (the reference GPU path truncates to i32 fixed point instead).
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/xpbd_cuda.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

namespace xpbd {

constexpr unsigned kFullMask = 0xFFFFFFFFu;
constexpr float kCollisionApplyClamp = 0.35f;  // COLLISION_APPLY_CLAMP, cloth_compute.rs:90

// ---------------------------------------------------------------------------------------------- hash keys
__device__ __forceinline__ int3 cell_of(float4 p, float inv_cell) {
    return make_int3((int)floorf(__fmul_rn(p.x, inv_cell)), (int)floorf(__fmul_rn(p.y, inv_cell)),
                     (int)floorf(__fmul_rn(p.z, inv_cell)));
}
__device__ __forceinline__ uint32_t hash_cell(int3 c, uint32_t mask) {
    return (((uint32_t)c.x * 73856093u) ^ ((uint32_t)c.y * 19349663u) ^ ((uint32_t)c.z * 83492791u)) & mask;
}

// With a bucket table: also marks empty the entries of the previous build's keys (still in `prev_sorted`, which
// the sort that follows overwrites), so that every valid-looking entry belongs to the current build.
__global__ void hash_keys_kernel(const float4* __restrict__ x, uint32_t n, float inv_cell, uint32_t mask,
                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                 const uint32_t* __restrict__ prev_sorted, uint2* __restrict__ table) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (table) table[prev_sorted[i]] = make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
        keys[i] = hash_cell(cell_of(x[i], inv_cell), mask);
        if (vals) vals[i] = i;
    }
}

// ---------------------------------------------------------------------------------------------- radix sort
// Per pass (8-bit digit): per-tile digit histogram → one exclusive scan over the digit-major (digit, tile)
// counts → stable scatter. Tile = 8 warps × 8 rounds × 32 keys; within a tile the order is warp, round, lane.
constexpr int kSortBlock = 256;
constexpr int kSortItems = 8;
constexpr uint32_t kSortTile = kSortBlock * kSortItems;

__global__ void __launch_bounds__(kSortBlock) radix_hist_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                 uint32_t shift, uint32_t tiles,
                                                                 uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        uint32_t idx = base + r * kSortBlock + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    counts[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Single-block exclusive scan of `m` u32 values in place, in chunks of 32768: thread t holds 8 rows of 4 consecutive
// values (row k starts at chunk + 4096k + 4t), so one chunk is one round of coalesced 16-byte loads. The 8 rows are
// scanned side by side: warp shuffles within each row, one shared-memory pass over the warps' row sums, and a running
// carry over rows and chunks. Launch with 1024 threads.
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanRows = 8;
constexpr uint32_t kScanChunk = kScanThreads * 4 * kScanRows;
__global__ void __launch_bounds__(kScanThreads) exclusive_scan_kernel(uint32_t* __restrict__ a, uint32_t m,
                                                                      uint32_t* __restrict__ total) {
    __shared__ uint32_t ws[kScanRows][32];  // warps' row sums, then their exclusive prefixes
    __shared__ uint32_t rowtot[kScanRows];
    const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
    const bool vec = (reinterpret_cast<uintptr_t>(a) & 15u) == 0;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < m; base += kScanChunk) {
        uint4 v[kScanRows];
#pragma unroll
        for (uint32_t k = 0; k < kScanRows; ++k) {
            const uint32_t i = base + k * (4 * kScanThreads) + 4 * t;
            if (vec && i + 3 < m && i + 3 > i) {
                v[k] = *reinterpret_cast<const uint4*>(a + i);
            } else {
                v[k].x = i < m ? a[i] : 0u;
                v[k].y = i + 1 < m ? a[i + 1] : 0u;
                v[k].z = i + 2 < m ? a[i + 2] : 0u;
                v[k].w = i + 3 < m ? a[i + 3] : 0u;
            }
        }
        uint32_t incl[kScanRows];
#pragma unroll
        for (uint32_t k = 0; k < kScanRows; ++k) incl[k] = v[k].x + v[k].y + v[k].z + v[k].w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (uint32_t k = 0; k < kScanRows; ++k) {
                const uint32_t x = __shfl_up_sync(kFullMask, incl[k], o);
                if (lane >= (uint32_t)o) incl[k] += x;
            }
        }
        if (lane == 31) {
#pragma unroll
            for (uint32_t k = 0; k < kScanRows; ++k) ws[k][warp] = incl[k];
        }
        __syncthreads();
        if (warp < kScanRows) {
            const uint32_t w = ws[warp][lane];
            uint32_t inc2 = w;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t x = __shfl_up_sync(kFullMask, inc2, o);
                if (lane >= (uint32_t)o) inc2 += x;
            }
            ws[warp][lane] = inc2 - w;
            if (lane == 31) rowtot[warp] = inc2;
        }
        __syncthreads();
#pragma unroll
        for (uint32_t k = 0; k < kScanRows; ++k) {
            const uint32_t i = base + k * (4 * kScanThreads) + 4 * t;
            const uint32_t sum = v[k].x + v[k].y + v[k].z + v[k].w;
            const uint32_t ex = carry + ws[k][warp] + incl[k] - sum;
            const uint4 o = make_uint4(ex, ex + v[k].x, ex + v[k].x + v[k].y, ex + v[k].x + v[k].y + v[k].z);
            if (vec && i + 3 < m && i + 3 > i) {
                *reinterpret_cast<uint4*>(a + i) = o;
            } else {
                if (i < m) a[i] = o.x;
                if (i + 1 < m) a[i + 1] = o.y;
                if (i + 2 < m) a[i + 2] = o.z;
                if (i + 3 < m) a[i + 3] = o.w;
            }
            carry += rowtot[k];
        }
        __syncthreads();  // ws and rowtot are rewritten by the next chunk
        if (base + kScanChunk < base) break;
    }
    if (total && t == 0) *total = carry;
}

__global__ void __launch_bounds__(kSortBlock) radix_scatter_kernel(const uint32_t* __restrict__ keys_in,
                                                                    const uint32_t* __restrict__ vals_in,
                                                                    uint32_t* __restrict__ keys_out,
                                                                    uint32_t* __restrict__ vals_out, uint32_t n,
                                                                    uint32_t shift, uint32_t tiles,
                                                                    const uint32_t* __restrict__ offsets) {
    __shared__ uint32_t s_wcnt[kSortBlock / 32][256];
    __shared__ uint32_t s_base[256];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint32_t k = threadIdx.x; k < (kSortBlock / 32) * 256; k += kSortBlock) (&s_wcnt[0][0])[k] = 0;
    __syncthreads();
    const uint32_t lanemask_lt = (1u << lane) - 1u;
    const uint32_t wbase = blockIdx.x * kSortTile + warp * (32 * kSortItems);
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        const bool valid = idx < n;
        key[r] = valid ? keys_in[idx] : 0u;
        val[r] = valid ? vals_in[idx] : 0u;
        const uint32_t d = valid ? ((key[r] >> shift) & 0xFFu) : 0x100u;
        const uint32_t peers = __match_any_sync(kFullMask, d);
        uint32_t before = 0;
        if (valid) before = s_wcnt[warp][d];
        __syncwarp();
        if (valid && lane == (uint32_t)(__ffs(peers) - 1)) s_wcnt[warp][d] = before + __popc(peers);
        __syncwarp();
        rank[r] = valid ? before + __popc(peers & lanemask_lt) : 0xFFFFFFFFu;
    }
    __syncthreads();
    {  // exclusive prefix over warps, per digit; tile base from the global scan
        const uint32_t d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortBlock / 32; ++w) {
            uint32_t t = s_wcnt[w][d];
            s_wcnt[w][d] = run;
            run += t;
        }
        s_base[d] = offsets[d * tiles + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        if (rank[r] == 0xFFFFFFFFu) continue;
        const uint32_t d = (key[r] >> shift) & 0xFFu;
        const uint32_t pos = s_base[d] + s_wcnt[warp][d] + rank[r];
        if (pos < n) {
            keys_out[pos] = key[r];
            vals_out[pos] = val[r];
        }
    }
}

cudaError_t launch_exclusive_scan(uint32_t* a, uint32_t m, uint32_t* total, cudaStream_t st) {
    if (m == 0) return cudaSuccess;
    exclusive_scan_kernel<<<1, kScanThreads, 0, st>>>(a, m, total);
    return cudaGetLastError();
}

size_t radix_sort_scratch_bytes(uint32_t n) {
    if (n > XPBD_RADIX_SORT_MAX_KEYS) return 0;
    size_t tiles = ((size_t)n + kSortTile - 1) / kSortTile;
    if (tiles == 0) tiles = 1;
    size_t counts = 256 * tiles * sizeof(uint32_t);
    size_t tmp = 2 * (size_t)n * sizeof(uint32_t);  // ping-pong keys/vals for even pass counts
    return ((counts + 255) & ~(size_t)255) + ((tmp + 255) & ~(size_t)255) + 256;
}

cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t n, uint32_t passes, void* scratch, size_t scratch_bytes,
                             cudaStream_t st, uint64_t* launches) {
    if (passes < 1 || passes > 4 || n > XPBD_RADIX_SORT_MAX_KEYS) return cudaErrorInvalidValue;
    if (n == 0) return cudaSuccess;
    if (scratch_bytes < radix_sort_scratch_bytes(n)) return cudaErrorInvalidValue;
    const uint32_t tiles = (uint32_t)(((size_t)n + kSortTile - 1) / kSortTile);  // <= 2^20 for n <= 2^31
    size_t counts_bytes = ((256 * (size_t)tiles * sizeof(uint32_t)) + 255) & ~(size_t)255;
    uint32_t* counts = (uint32_t*)scratch;
    uint32_t* tmp_k = (uint32_t*)((char*)scratch + counts_bytes);
    uint32_t* tmp_v = tmp_k + n;
    // choose ping-pong so that the last pass writes keys_out/vals_out
    const uint32_t* src_k = keys_in;
    const uint32_t* src_v = vals_in;
    for (uint32_t p = 0; p < passes; ++p) {
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        uint32_t* dk = to_out ? keys_out : tmp_k;
        uint32_t* dv = to_out ? vals_out : tmp_v;
        const uint32_t shift = 8u * p;
        radix_hist_kernel<<<tiles, kSortBlock, 0, st>>>(src_k, n, shift, tiles, counts);
        exclusive_scan_kernel<<<1, kScanThreads, 0, st>>>(counts, 256 * tiles, nullptr);
        radix_scatter_kernel<<<tiles, kSortBlock, 0, st>>>(src_k, src_v, dk, dv, n, shift, tiles, counts);
        if (launches) *launches += 3;
        src_k = dk;
        src_v = dv;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- sort, no allocation
// Scratch of the allocation-free sort: a file-scope device array sized for XPBD_NOALLOC_SORT_MAX_KEYS keys (per-tile
// digit counts + the ping-pong key/value buffers), held by every GPU that loads the library until the process exits.
constexpr size_t noalloc_scratch_bytes(uint32_t n) {
    return ((256 * (size_t)((n + kSortTile - 1) / kSortTile) * sizeof(uint32_t) + 255) & ~(size_t)255) +
           ((2 * (size_t)n * sizeof(uint32_t) + 255) & ~(size_t)255) + 256;
}
constexpr size_t kNoAllocScratchBytes = noalloc_scratch_bytes(XPBD_NOALLOC_SORT_MAX_KEYS);
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocScratchBytes];

// Identity of the current context (cuCtxGetId: unique over the process's lifetime, never reused), through the
// runtime's driver entry points so that the library does not link libcuda; 0 when unavailable.
static unsigned long long current_context_id() {
    typedef int (*CtxGetCurrent)(void**);
    typedef int (*CtxGetId)(void*, unsigned long long*);
    static CtxGetCurrent get_current = nullptr;
    static CtxGetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetId)f;
    });
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array in the current context. The array's name is only a host-side stand-in, so the
// address is looked up with the device current and cached per device together with the context it belongs to; a
// re-created context (after cudaDeviceReset) gets a fresh lookup.
static cudaError_t noalloc_scratch(void** out) {
    static std::mutex mu;
    static void* cache[64] = {nullptr};
    static unsigned long long cache_ctx[64] = {0};
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_context_id();  // 0 before the runtime made a context current
    if (!cache[dev] || ctx == 0 || cache_ctx[dev] != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);  // makes the device's context current if needed
        if (e != cudaSuccess) return e;
        cache[dev] = p;
        cache_ctx[dev] = current_context_id();
    }
    *out = cache[dev];
    return cudaSuccess;
}

cudaError_t launch_hash_keys(const float4* x, uint32_t n, float inv_cell, uint32_t bits, uint32_t* keys,
                             uint32_t* vals, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t grid = (n + 255) / 256;
    if (grid > 148u * 16u) grid = 148u * 16u;
    hash_keys_kernel<<<grid, 256, 0, st>>>(x, n, inv_cell, (bits >= 32) ? 0xFFFFFFFFu : ((1u << bits) - 1u), keys,
                                           vals, nullptr, nullptr);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- bucket table
// Bucket ranges of the sorted keys, and the positions gathered into sorted order so that the candidates of a bucket
// are read from consecutive addresses.
__global__ void bucket_table_kernel(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ svals,
                                    const float4* __restrict__ pos, uint32_t n, uint2* __restrict__ table,
                                    float4* __restrict__ pos_sorted) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t k = skeys[p];
        if (p == 0 || skeys[p - 1] != k) table[k].x = p;
        if (p + 1 == n || skeys[p + 1] != k) table[k].y = p + 1;
        pos_sorted[p] = pos[svals[p]];
    }
}

cudaError_t collision_build(const XpbdWorld& W, const float4* pos, const CollisionBuffers& B, float inv_cell,
                            int sms, cudaStream_t st, uint64_t* launches) {
    if (W.n > 0) {
        uint32_t g = (W.n + 255) / 256;
        if (g > 148u * 16u) g = 148u * 16u;
        hash_keys_kernel<<<g, 256, 0, st>>>(pos, W.n, inv_cell,
                                            (B.table_bits >= 32) ? 0xFFFFFFFFu : ((1u << B.table_bits) - 1u), B.keys,
                                            B.vals, B.keys_sorted, B.table);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // Keys are below 2^table_bits: the passes over the all-zero high digits would be identity permutations.
    uint32_t passes = B.table_bits >= 32 ? 4u : (B.table_bits + 7u) / 8u;
    if (passes < 1u) passes = 1u;
    e = radix_sort_pairs(B.keys, B.vals, B.keys_sorted, B.vals_sorted, W.n, passes, B.sort_scratch,
                         B.sort_scratch_bytes, st, launches);
    if (e != cudaSuccess) return e;
    uint32_t grid = (W.n + 255) / 256;
    if (grid > (uint32_t)sms * 8) grid = (uint32_t)sms * 8;
    if (grid == 0) grid = 1;
    bucket_table_kernel<<<grid, 256, 0, st>>>(B.keys_sorted, B.vals_sorted, pos, W.n, B.table, B.pos_sorted);
    if (launches) *launches += 2;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- narrow phase
struct F3c {
    float x, y, z;
};
__device__ __forceinline__ float dot3c(F3c a, F3c b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}

__device__ __forceinline__ bool ring_contains(const uint32_t* __restrict__ off, const uint32_t* __restrict__ idx,
                                              uint32_t a, uint32_t b) {
    uint32_t lo = off[a], hi = off[a + 1];
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t v = idx[mid];
        if (v == b) return true;
        if (v < b) lo = mid + 1; else hi = mid;
    }
    return false;
}

// Pair (a<b) narrow phase of xpbd_cpu.rs:84-121 (filter 1: rest-distance test :94-100; filter 2: ring filter), on
// the positions pa, pb of a, b. On acceptance returns the correction of particle `self` (a or b).
__device__ __forceinline__ bool narrow_pair(const float4 pa, const float4 pb, const float4* __restrict__ rest,
                                            const CollisionBuffers& B, uint32_t filter, float thickness,
                                            float coll_scale, uint32_t a, uint32_t b, uint32_t self, F3c& out) {
    const float w_a = pa.w, w_b = pb.w;
    if (w_a <= 0.0f && w_b <= 0.0f) return false;
    const float t2 = __fmul_rn(thickness, thickness);
    F3c d = {__fsub_rn(pb.x, pa.x), __fsub_rn(pb.y, pa.y), __fsub_rn(pb.z, pa.z)};
    const float dist2 = dot3c(d, d);
    if (dist2 > t2 || dist2 < 1e-18f) return false;
    const float4 ra = rest[a], rb = rest[b];
    const F3c rd = {__fsub_rn(rb.x, ra.x), __fsub_rn(rb.y, ra.y), __fsub_rn(rb.z, ra.z)};
    const float rest2 = dot3c(rd, rd);
    if (filter == 1u) {
        if (dist2 > rest2) return false;
    } else if (ring_contains(B.ring_off, B.ring_idx, a, b)) {
        return false;
    }
    float min_d = thickness;
    if (rest2 < t2) min_d = __fsqrt_rn(rest2);
    const float dist = __fsqrt_rn(dist2);
    const float corr = __fmul_rn(__fmul_rn(__fsub_rn(min_d, dist), 0.5f), coll_scale);
    if (corr <= 0.0f) return false;
    d = {__fmul_rn(__fdiv_rn(d.x, dist), corr), __fmul_rn(__fdiv_rn(d.y, dist), corr),
         __fmul_rn(__fdiv_rn(d.z, dist), corr)};
    const float inv_w = __fdiv_rn(1.0f, fmaxf(__fadd_rn(w_a, w_b), 1e-8f));
    if (self == a)
        out = {__fmul_rn(__fmul_rn(-d.x, w_a), inv_w), __fmul_rn(__fmul_rn(-d.y, w_a), inv_w),
               __fmul_rn(__fmul_rn(-d.z, w_a), inv_w)};
    else
        out = {__fmul_rn(__fmul_rn(d.x, w_b), inv_w), __fmul_rn(__fmul_rn(d.y, w_b), inv_w),
               __fmul_rn(__fmul_rn(d.z, w_b), inv_w)};
    return true;
}

// Squared gaps, in cell units, from u = fl(p·inv_cell) to the lower and upper faces of its cell (f = floor(u)), each
// shortened by a slack of (2|u| + reach + 2)·2^-20: eight times the rounding of u for both particles of a pair
// (2^-23·|u| each) and of the gap itself.
__device__ __forceinline__ void cell_face_gaps(float u, float f, float reach, float& lo2, float& hi2) {
    const float slack = __fmul_rn(__fadd_rn(__fadd_rn(__fmul_rn(2.0f, fabsf(u)), reach), 2.0f), 0x1p-20f);
    const float lo = fmaxf(__fsub_rn(__fsub_rn(u, f), slack), 0.0f);
    const float hi = fmaxf(__fsub_rn(__fsub_rn(__fadd_rn(f, 1.0f), u), slack), 0.0f);
    lo2 = __fmul_rn(lo, lo);
    hi2 = __fmul_rn(hi, hi);
}

// Visits every particle j != i, with its position, in the (deduplicated) buckets of the 27 cells around i's cell,
// leaving out the cells that hold no particle within `thickness` of i. The narrow phase accepts only pairs at most
// `thickness` apart, so when thickness is below the cell size (every accepted partner then lies in one of the 27
// cells) the accepted partners are the same; a left-out cell is not marked as seen, so its bucket is still visited
// through any other cell that hashes to it. Partners are summed in index order, so the visiting order does not
// change a result.
template <typename F>
__device__ __forceinline__ void for_each_candidate(const float4* __restrict__ src, const CollisionBuffers& B,
                                                   uint32_t n, uint32_t i, float inv_cell, float thickness, F&& f) {
    const uint32_t mask = (B.table_bits >= 32) ? 0xFFFFFFFFu : ((1u << B.table_bits) - 1u);
    const float4 p = src[i];
    const float ux = __fmul_rn(p.x, inv_cell), uy = __fmul_rn(p.y, inv_cell), uz = __fmul_rn(p.z, inv_cell);
    const float fx = floorf(ux), fy = floorf(uy), fz = floorf(uz);
    const int3 c = make_int3((int)fx, (int)fy, (int)fz);  // == cell_of(p, inv_cell)
    // Reach of the narrow phase in cell units; the gap test runs only while it is below one cell (NaN: never).
    const float reach = fabsf(__fmul_rn(thickness, inv_cell));
    const float reach2 = reach < 0.999f ? __fmul_rn(__fmul_rn(reach, reach), 1.001f) : __int_as_float(0x7f800000);
    float xlo2, xhi2, ylo2, yhi2, zlo2, zhi2;
    cell_face_gaps(ux, fx, reach, xlo2, xhi2);
    cell_face_gaps(uy, fy, reach, ylo2, yhi2);
    cell_face_gaps(uz, fz, reach, zlo2, zhi2);
    uint32_t seen[27];
    int nseen = 0;
    for (int dz = -1; dz <= 1; ++dz) {
        const float gz = dz < 0 ? zlo2 : (dz > 0 ? zhi2 : 0.0f);
        for (int dy = -1; dy <= 1; ++dy) {
            const float gyz = __fadd_rn(gz, dy < 0 ? ylo2 : (dy > 0 ? yhi2 : 0.0f));
            for (int dx = -1; dx <= 1; ++dx) {
                if (__fadd_rn(gyz, dx < 0 ? xlo2 : (dx > 0 ? xhi2 : 0.0f)) > reach2) continue;
                const uint32_t h = hash_cell(make_int3(c.x + dx, c.y + dy, c.z + dz), mask);
                bool dup = false;
                for (int q = 0; q < nseen; ++q) dup |= (seen[q] == h);
                if (dup) continue;
                seen[nseen++] = h;
                // entries of buckets absent from this build were marked empty by it (hash_keys_kernel)
                const uint2 t = B.table[h];
                const uint32_t s = t.x;
                if (s >= n) continue;
                const uint32_t e = min(t.y, n);
                for (uint32_t q = s; q < e; ++q) {
                    const uint32_t j = B.vals_sorted[q];
                    const float4 pj = B.pos_sorted[q];
                    if (j != i) f(j, pj);
                }
            }
        }
    }
}

constexpr int kPartnerCap = 24;

// Accepted partners of i with index in (lo, ∞), the kPartnerCap smallest, sorted. Returns true if more remain.
template <bool ONLY_GREATER>
__device__ __forceinline__ bool collect_partners(const float4* __restrict__ src, const float4* __restrict__ rest,
                                                 const CollisionBuffers& B, uint32_t n, uint32_t i, float inv_cell,
                                                 uint32_t filter, float thickness, float coll_scale, long long lo,
                                                 uint32_t* pj, F3c* pc, int& cnt) {
    cnt = 0;
    bool overflow = false;
    const float4 p_i = src[i];
    for_each_candidate(src, B, n, i, inv_cell, thickness, [&](uint32_t j, const float4 p_j) {
        if ((long long)j <= lo) return;
        if (ONLY_GREATER && j < i) return;
        const bool i_first = i < j;
        const uint32_t a = i_first ? i : j, b = i_first ? j : i;
        const float4 pa = i_first ? p_i : p_j, pb = i_first ? p_j : p_i;
        if (cnt == kPartnerCap && j > pj[kPartnerCap - 1]) {
            // cheap reject before the narrow test; it may be accepted, so remember that more partners remain
            F3c tmp;
            if (narrow_pair(pa, pb, rest, B, filter, thickness, coll_scale, a, b, i, tmp)) overflow = true;
            return;
        }
        F3c corr;
        if (!narrow_pair(pa, pb, rest, B, filter, thickness, coll_scale, a, b, i, corr)) return;
        if (cnt == kPartnerCap) overflow = true;  // evicts the largest
        int p = (cnt < kPartnerCap) ? cnt++ : kPartnerCap - 1;
        while (p > 0 && pj[p - 1] > j) {
            pj[p] = pj[p - 1];
            pc[p] = pc[p - 1];
            --p;
        }
        pj[p] = j;
        pc[p] = corr;
    });
    return overflow;
}

// collide: dst[i] = src[i] + clamp(Σ_j corr_ij) with partners in increasing index (xpbd_cpu.rs:82-136).
// 16 blocks of 128 per SM (32 registers): one thread per particle then fits in a single wave for a 262k-particle
// sheet; the latency-bound walk gains more from the extra resident warps than it loses to the few spills.
__global__ void __launch_bounds__(128, 16) collision_resolve_kernel(XpbdWorld W, const float4* __restrict__ src,
                                                                float4* __restrict__ dst, CollisionBuffers B,
                                                                float inv_cell, uint32_t filter) {
    const XpbdDevParams& P = *W.params;
    const float thickness = P.thickness, coll_scale = P.coll_scale;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < W.n; p += gridDim.x * blockDim.x) {
        const uint32_t i = p;  // mesh order: neighbouring threads query overlapping cells
        const float4 pi = src[i];
        if (pi.w <= 0.0f) {
            dst[i] = pi;
            continue;
        }
        uint32_t pj[kPartnerCap];
        F3c pc[kPartnerCap];
        F3c acc = {0.0f, 0.0f, 0.0f};
        long long lo = -1;
        for (int round = 0; round < 1 << 16; ++round) {
            int cnt = 0;
            const bool more = collect_partners<false>(src, W.rest, B, W.n, i, inv_cell, filter, thickness,
                                                      coll_scale, lo, pj, pc, cnt);
            for (int q = 0; q < cnt; ++q) {
                acc.x = __fadd_rn(acc.x, pc[q].x);
                acc.y = __fadd_rn(acc.y, pc[q].y);
                acc.z = __fadd_rn(acc.z, pc[q].z);
            }
            if (!more || cnt == 0) break;
            lo = pj[cnt - 1];
        }
        const float m = kCollisionApplyClamp;
        const float cx = fminf(fmaxf(acc.x, -m), m), cy = fminf(fmaxf(acc.y, -m), m), cz = fminf(fmaxf(acc.z, -m), m);
        dst[i] = make_float4(__fadd_rn(pi.x, cx), __fadd_rn(pi.y, cy), __fadd_rn(pi.z, cz), pi.w);
    }
}

cudaError_t collision_resolve(const XpbdWorld& W, const float4* src, float4* dst, const CollisionBuffers& B,
                              float inv_cell, uint32_t filter, int sms, cudaStream_t st, uint64_t* launches) {
    uint32_t grid = (W.n + 127) / 128;
    if (grid > (uint32_t)sms * 16) grid = (uint32_t)sms * 16;
    if (grid == 0) grid = 1;
    collision_resolve_kernel<<<grid, 128, 0, st>>>(W, src, dst, B, inv_cell, filter);
    if (launches) *launches += 1;
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------------- pair list
__global__ void pair_count_kernel(XpbdWorld W, const float4* __restrict__ src, CollisionBuffers B, float inv_cell,
                                  uint32_t filter, uint32_t* __restrict__ counts) {
    const XpbdDevParams& P = *W.params;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n; i += gridDim.x * blockDim.x) {
        uint32_t c = 0;
        const float4 p_i = src[i];
        for_each_candidate(src, B, W.n, i, inv_cell, P.thickness, [&](uint32_t j, const float4 p_j) {
            if (j < i) return;
            F3c tmp;
            if (narrow_pair(p_i, p_j, W.rest, B, filter, P.thickness, P.coll_scale, i, j, i, tmp)) ++c;
        });
        counts[i] = c;
    }
}

__global__ void pair_write_kernel(XpbdWorld W, const float4* __restrict__ src, CollisionBuffers B, float inv_cell,
                                  uint32_t filter, const uint32_t* __restrict__ offsets, uint32_t* __restrict__ out,
                                  unsigned long long cap) {
    const XpbdDevParams& P = *W.params;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < W.n; i += gridDim.x * blockDim.x) {
        uint32_t pj[kPartnerCap];
        F3c pc[kPartnerCap];
        unsigned long long o = offsets[i];
        long long lo = -1;
        for (int round = 0; round < 1 << 16; ++round) {
            int cnt = 0;
            const bool more = collect_partners<true>(src, W.rest, B, W.n, i, inv_cell, filter, P.thickness,
                                                     P.coll_scale, lo, pj, pc, cnt);
            for (int q = 0; q < cnt; ++q, ++o)
                if (o < cap) {
                    out[2 * o] = i;
                    out[2 * o + 1] = pj[q];
                }
            if (!more || cnt == 0) break;
            lo = pj[cnt - 1];
        }
    }
}

cudaError_t collision_pairs(const XpbdWorld& W, const float4* pos, const CollisionBuffers& B, float inv_cell,
                            uint32_t filter, uint32_t* pairs_out, uint64_t cap, uint64_t* total, int sms,
                            cudaStream_t st) {
    uint32_t grid = (W.n + 127) / 128;
    if (grid > (uint32_t)sms * 16) grid = (uint32_t)sms * 16;
    if (grid == 0) grid = 1;
    pair_count_kernel<<<grid, 128, 0, st>>>(W, pos, B, inv_cell, filter, B.pair_count);
    cudaError_t e = cudaMemsetAsync(B.pair_count + W.n, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    exclusive_scan_kernel<<<1, kScanThreads, 0, st>>>(B.pair_count, W.n + 1, nullptr);
    uint32_t h_total = 0;
    e = cudaMemcpyAsync(&h_total, B.pair_count + W.n, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    *total = h_total;
    if (pairs_out && cap > 0) pair_write_kernel<<<grid, 128, 0, st>>>(W, pos, B, inv_cell, filter, B.pair_count,
                                                                      pairs_out, cap);
    return cudaGetLastError();
}

}  // namespace xpbd

// True when the output arrays of a sort of n keys overlap each other or an input array.
bool xpbd_sort_arrays_overlap(const void* keys_in, const void* vals_in, const void* keys_out, const void* vals_out,
                              uint32_t n) {
    const uintptr_t b = 4 * (uintptr_t)n;
    auto meet = [b](const void* p, const void* q) {
        const uintptr_t a = (uintptr_t)p, c = (uintptr_t)q;
        return a < c + b && c < a + b;
    };
    return meet(keys_out, vals_out) || meet(keys_out, keys_in) || meet(keys_out, vals_in) ||
           meet(vals_out, keys_in) || meet(vals_out, vals_in);
}

extern "C" int xpbd_radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                             uint32_t* vals_out, uint32_t n, uint32_t passes, void* stream) {
    if (n && (!keys_in || !vals_in || !keys_out || !vals_out)) return XPBD_ERR_INVALID_ARGUMENT;
    if (passes < 1 || passes > 4) return XPBD_ERR_INVALID_ARGUMENT;
    if (n && xpbd_sort_arrays_overlap(keys_in, vals_in, keys_out, vals_out, n)) return XPBD_ERR_INVALID_ARGUMENT;
    if (n > XPBD_NOALLOC_SORT_MAX_KEYS) return XPBD_ERR_CAPACITY;
    if (n == 0) return XPBD_OK;
    void* scratch = nullptr;
    if (xpbd::noalloc_scratch(&scratch) != cudaSuccess) return XPBD_ERR_CUDA;
    // nothing in the scratch must start at zero: each pass writes every digit count and every ping-pong word
    // before reading it, so the previous call's contents are harmless
    cudaError_t e = xpbd::radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, passes, scratch,
                                           xpbd::kNoAllocScratchBytes, (cudaStream_t)stream, nullptr);
    return e == cudaSuccess ? XPBD_OK : XPBD_ERR_CUDA;
}
