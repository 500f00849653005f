// Host-side launchers of the sm_100a kernels (solver_kernels.cu, collision_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "xpbd_internal.h"

namespace xpbd {

constexpr uint32_t kBeginFinalize = 1u;  // finalize positions waiting in jac[pend] before predicting
constexpr uint32_t kEndFinalize = 2u;    // finalize the launch's last substep in place

// ---- solver (solver_kernels.cu); kernel id: 0 Jacobi warp tiles, 1 Gauss–Seidel, 2 Jacobi spatial patches,
//      5 Jacobi thread per particle, 6 Jacobi convergence solve
const void* solver_kernel_fn(uint32_t solver, uint32_t block);
int max_blocks_per_sm(uint32_t solver, uint32_t block, const XpbdWorld& W);
cudaError_t launch_solver(uint32_t solver, uint32_t block, uint32_t grid, bool cooperative, const XpbdWorld& W,
                          uint32_t flags, uint32_t substeps, uint32_t pend, uint32_t start, cudaStream_t st);
cudaError_t launch_finalize(const XpbdWorld& W, uint32_t pend, int sms, cudaStream_t st);
cudaError_t launch_converge_predict(const XpbdWorld& W, int sms, cudaStream_t st);
cudaError_t launch_strain_residual(const XpbdWorld& W, uint32_t e0, uint32_t e1, unsigned* out_bits, int sms,
                                   cudaStream_t st);

cudaError_t launch_vertex_normals(const XpbdWorld& W, int sms, cudaStream_t st);
cudaError_t launch_division_selftest(uint64_t count, uint64_t seed, unsigned long long* mismatches, int sms,
                                     cudaStream_t st);

// ---- warm-start MLP (mlp.cu)
cudaError_t launch_mlp_infer(const XpbdWorld& W, const XpbdMlp* mlp, int sms, cudaStream_t st);
cudaError_t launch_mlp_eval(const XpbdMlp* mlp, const float* feat, uint32_t n, float* out, cudaStream_t st);
cudaError_t launch_mlp_collect_features(const XpbdWorld& W, uint32_t stride, uint32_t offset, float* feat,
                                        float* scale, uint32_t base, uint32_t cap, cudaStream_t st);
cudaError_t launch_mlp_collect_targets(const XpbdWorld& W, uint32_t stride, uint32_t offset, const float* scale,
                                       float* target, uint32_t base, uint32_t cap, cudaStream_t st);
// One training step's gradient (tcgen05 tensor cores): grads += d loss / d params over rows idx[0..nrows), loss += Σ e²;
// a tensor-core wait that gives up sets XPBD_DEV_BARRIER_TIMEOUT in *status.
cudaError_t launch_mlp_train(const XpbdMlp* mlp, const float* feat, const float* target, const uint32_t* idx,
                             uint32_t nrows, float* grads, float* loss, int* status, cudaStream_t st);
cudaError_t launch_mlp_adam(float* master, float* m1, float* m2, const float* grads, float gscale, float lr,
                            float beta1, float beta2, float eps, float bc1, float bc2, XpbdMlp* mlp, cudaStream_t st);
cudaError_t launch_mlp_publish(const float* master, XpbdMlp* mlp, cudaStream_t st);

// ---- cloth-resident Jacobi (cloth_jacobi.cu)
struct ClothSolveTable {
    const XpbdClothDesc* cloths;  // per cloth of the batch
    const uint32_t* seg;          // (color, rank) segment starts into rec / comp
    const uint2* rec;             // {endpoint i | endpoint j << 16, rest bits}
    const float* comp;            // compliance per record
    const uint32_t* order;        // cloth ids of one launch (one per cluster), largest first
    uint32_t count;               // cloths in the launch
    uint32_t cap;                 // shared-memory slots per rank in this launch (>= every cloth's q)
};
// Launch shapes of the cloth-resident kernel: CTAs per cluster and threads per CTA; a cloth of n particles takes
// the first class whose capacity (cl x per-rank slots) holds it.
struct ClothClass {
    uint32_t cl, block, rank_cap;
};
constexpr int kClothClasses = 7;
extern const ClothClass kClothClass[kClothClasses];
size_t cloth_kernel_smem_bytes(uint32_t cap);
cudaError_t launch_cloth_jacobi(int cls, const XpbdWorld& W, const ClothSolveTable& T, uint32_t substeps,
                               cudaStream_t st);
cudaError_t cloth_kernel_prepare();  // opt-in shared-memory sizes (host, once)
bool cloth_class_launchable(int cls);  // a cluster of the class fits on this device
// A whole small batch in one cluster of cl (8 or 16) CTAs, thread per incidence (cloth_jacobi.cu).
struct SmallBatch {
    const uint4* rec;       // rank-major records {self local | slot in its row << 16, other endpoint (local | rank << 12
                            // | slot in the other's row << 16 | 1 << 31 when that row is on the same rank: one record
                            // for both endpoints), rest, comp}
    const uint32_t* roff;   // per rank: q + 1 local row starts (prefix sums of the row lengths)
    const uint32_t* rbase;  // cl + 1: first record of each rank in rec
    uint32_t q;             // particles per rank
    uint32_t m_max;         // largest record count of a rank
    uint32_t stride;        // term slots per row in shared memory: 4·ceil(longest row / 4) + 1 (odd)
};
size_t small_batch_smem_bytes(uint32_t q, uint32_t m_max, uint32_t stride);
bool small_batch_supported(uint32_t cl, uint32_t block, uint32_t q, uint32_t m_max, uint32_t stride);
cudaError_t launch_small_batch(uint32_t cl, uint32_t block, const XpbdWorld& W, const SmallBatch& B,
                               uint32_t substeps, cudaStream_t st);

// ---- Gauss–Seidel over several clusters (strip_gs.cu)
struct StripTable {
    const uint4* rec;        // {code i, code j, rest, comp} grouped by (color, CTA, kind 0/1/2)
    const uint32_t* off;     // 3 · ncolors · ncta + 1 group starts
    const uint32_t* slot;    // per particle: its global slot when shared between strips, else 0xFFFFFFFF
    float4* gx;              // shared particles' positions during a frame
    unsigned* flags;         // per CTA: steps completed (monotonic across launches)
    const uint32_t* deps;    // CTAs of other strips sharing particles with a CTA, dep_off[cta] .. dep_off[cta + 1]
    const uint32_t* dep_off;
    uint32_t q, ncta, ncolors;
};
size_t strip_gs_smem_bytes(uint32_t q);
bool strip_gs_supported(uint32_t cl, uint32_t strips, uint32_t block, uint32_t q);
cudaError_t launch_strip_gs(uint32_t cl, uint32_t block, const XpbdWorld& W, const StripTable& T, uint32_t substeps,
                            cudaStream_t st);

// ---- cluster Gauss–Seidel (cluster_gs.cu)
// Shared-memory slot of a CTA's local particle p in the cluster Gauss–Seidel kernel: bits 3-5 of p flip its low
// three bits, a bijection within every 64 slots that spreads the particles one color touches (often every other one
// along a row) over the eight 16-byte bank groups.
__host__ __device__ __forceinline__ uint32_t cluster_slot(uint32_t p) { return p ^ ((p >> 3) & 7u); }
struct ClusterTable {
    const uint4* rec;    // constraint records grouped by (color, owning rank); endpoints as rank << shift | slot
    const uint32_t* off; // ncolors * CL + 1 offsets into rec
    const uint32_t* nbd; // per (color, rank) group: leading records that touch a boundary particle
    uint32_t shift;      // particles per CTA = 1 << shift
    uint32_t max_chunk;  // largest (color, rank) group, in records
};
size_t cluster_gs_smem_bytes(uint32_t shift, uint32_t max_chunk);
bool cluster_gs_supported(uint32_t cl, uint32_t shift, uint32_t max_chunk, uint32_t block);
cudaError_t launch_cluster_gs(uint32_t cl, uint32_t block, const XpbdWorld& W, const ClusterTable& T, uint32_t flags,
                              uint32_t substeps, uint32_t pend, cudaStream_t st);

// ---- collision (collision_kernels.cu)
struct CollisionBuffers {
    uint32_t* keys;         // n
    uint32_t* vals;         // n
    uint32_t* keys_sorted;  // n
    uint32_t* vals_sorted;  // n
    uint2* table;           // 2^bits bucket -> {first, one past the last} sorted position; each build marks the
                            // previous build's buckets empty (0xFFFFFFFF) before writing its own
    float4* pos_sorted;     // n: the positions in sorted order, gathered by the bucket pass
    uint32_t* pair_count;   // n + 1 (pair extraction only)
    void* sort_scratch;
    size_t sort_scratch_bytes;
    uint32_t table_bits;
    const uint32_t* ring_off;  // n + 1 (ring filter)
    const uint32_t* ring_idx;
};
// Single-block exclusive scan of m u32 values in place; total (device, may be null) receives the sum.
cudaError_t launch_exclusive_scan(uint32_t* a, uint32_t m, uint32_t* total, cudaStream_t st);
size_t radix_sort_scratch_bytes(uint32_t n);
cudaError_t radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t n, uint32_t passes, void* scratch, size_t scratch_bytes,
                             cudaStream_t st, uint64_t* launches);
cudaError_t launch_hash_keys(const float4* x, uint32_t n, float inv_cell, uint32_t bits, uint32_t* keys,
                             uint32_t* vals, cudaStream_t st);
// Keys, sort and bucket table of the positions in `pos`.
cudaError_t collision_build(const XpbdWorld& W, const float4* pos, const CollisionBuffers& B, float inv_cell,
                            int sms, cudaStream_t st, uint64_t* launches);
// Self collision of `src` into `dst` (reference narrow phase, contributions summed in partner-index order).
cudaError_t collision_resolve(const XpbdWorld& W, const float4* src, float4* dst, const CollisionBuffers& B,
                              float inv_cell, uint32_t filter, int sms, cudaStream_t st, uint64_t* launches);
// Pair list (a<b, lexicographic). Two passes: count per particle, exclusive scan, write.
cudaError_t collision_pairs(const XpbdWorld& W, const float4* pos, const CollisionBuffers& B, float inv_cell,
                            uint32_t filter, uint32_t* pairs_out, uint64_t cap, uint64_t* total, int sms,
                            cudaStream_t st);

}  // namespace xpbd
