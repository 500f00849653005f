/*
 * xpbd_cuda.h — C ABI of the B200 (sm_100a) XPBD cloth substep.
 *
 * Drop-in boundary for the GPU driver of the Rust crate `bevy_softbody` (mate-h/bevy_xpbd). The crate keeps its
 * mesh preparation (src/mesh_prep.rs) and its plugin/resource types; what this library replaces is the wgpu host
 * driver (src/cloth_jacobi.rs, src/cloth_compute.rs) and its WGSL kernels (src/shaders/cloth_sim_jacobi.wgsl,
 * src/shaders/cloth_sim.wgsl). Each entry point below names the reference interface it stands in for.
 *
 * Conventions: plain pointers and sizes, no CUDA or torch types (streams are passed as `void*` holding a
 * cudaStream_t). Every function returns XPBD_OK (0) or a negative XPBD_ERR_* code; xpbd_last_error() gives the
 * message. Positions and velocities cross the boundary as packed xyz float triples (the reference's Vec3).
 * One context per host thread; a context owns its device buffers and its stream. Device-side failures (non-finite
 * positions, grid-barrier timeout, collision-list overflow, index out of range) are recorded in a device status
 * word and returned by the next call that synchronises (xpbd_sync, xpbd_read_*).
 */
#ifndef XPBD_CUDA_H
#define XPBD_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------------------- */
#define XPBD_OK 0
#define XPBD_ERR_INVALID_ARGUMENT (-1)
#define XPBD_ERR_CUDA (-2)
#define XPBD_ERR_OUT_OF_MEMORY (-3)
#define XPBD_ERR_UNSUPPORTED (-4)
#define XPBD_ERR_STATE (-5)
#define XPBD_ERR_DEVICE_NONFINITE (-6)
#define XPBD_ERR_BARRIER_TIMEOUT (-7)
#define XPBD_ERR_INDEX_RANGE (-8)
#define XPBD_ERR_CAPACITY (-9)
#define XPBD_ERR_NO_DEVICE (-10)

/* ---- enumerations ---------------------------------------------------------------------------------------- */
#define XPBD_SOLVER_JACOBI 0        /* Cargo feature solver-jacobi (default), cloth_jacobi.rs */
#define XPBD_SOLVER_GAUSS_SEIDEL 1  /* Cargo feature solver-gauss-seidel, cloth_compute.rs:1271-1522 */

#define XPBD_RELAX_OMEGA 0          /* Δx = ω·Σ (xpbd_cpu.rs:223, ω = jacobi_default_omega() = 0.32) */
#define XPBD_RELAX_AVERAGE 1        /* Δx = ω·Σ / (constraints at the particle) — no reference counterpart */

#define XPBD_LAMBDA_RESET_PER_ITERATION 0 /* λ cleared before every inner iteration (xpbd_cpu.rs:267) */
#define XPBD_LAMBDA_PER_SUBSTEP 1         /* λ cleared (or warm-started) once per substep — standard XPBD */

#define XPBD_COLLISION_NONE 0
#define XPBD_COLLISION_REST_FILTER 1 /* self_collision_resolve filter: skip if dist² > rest² (xpbd_cpu.rs:98) */
#define XPBD_COLLISION_RING_FILTER 2 /* skip partners within `ring_depth` topology rings (stretch+shear edges) */

#define XPBD_ORDER_COLOR_REFERENCE 0 /* recolor: partition_constraints_for_gs_batches order (mesh_prep.rs:172-177) */
#define XPBD_ORDER_COLOR_INDEX 1     /* recolor greedily in plain constraint-index order */
#define XPBD_ORDER_PRESORTED 2       /* constraints already batch-sorted by the caller; use its batch offsets */

#define XPBD_WARM_NONE 0      /* plain start: λ = 0, predicted positions */
#define XPBD_WARM_LEARNED 1   /* λ0 from the context's MLP (xpbd_mlp_*) */
#define XPBD_WARM_GIVEN 2     /* λ0 set with xpbd_set_warm_lambda */
#define XPBD_WARM_PREVIOUS 3  /* λ0 = the previous substep's final λ */

#define XPBD_CONSTRAINT_STRETCH 0
#define XPBD_CONSTRAINT_SHEAR 1
#define XPBD_CONSTRAINT_BEND 2

/* ---- parameter blocks ------------------------------------------------------------------------------------ */

/* XpbdCpuTimeStepParams (xpbd_cpu.rs:11-26); on the GPU side the same fields travel in ClothSimParamsGpu
 * (cloth_compute.rs:245-273), which this library derives (inv_dt², exp(-k·dt)) and uploads per call. */
typedef struct xpbd_time_step_params {
    float dt;                   /* substep length [s] */
    float inv_dt;
    float jacobi_omega;
    uint32_t inner_iterations;
    float gravity[3];
    int32_t grab_idx;           /* particle index within the context (cloth offsets added), -1 = none */
    uint32_t grab_active;
    float grab_target[3];
    float grab_stiffness;
    float linear_drag_per_sec;  /* v *= exp(-k·dt) per substep */
} xpbd_time_step_params;

/* Solver configuration: ClothSimConfig (cloth_compute.rs:140-179) + ClothSimUniforms collision fields
 * (:181-202), and the extension modes. Zero-initialise, then set what differs; xpbd_default_opts() fills the
 * reference defaults. */
typedef struct xpbd_solver_opts {
    uint32_t solver;                  /* XPBD_SOLVER_* */
    uint32_t relaxation;              /* XPBD_RELAX_* */
    uint32_t lambda_mode;             /* XPBD_LAMBDA_* */
    uint32_t substeps;                /* solve_substeps per frame */
    uint32_t collision;               /* XPBD_COLLISION_* */
    uint32_t collision_every_n_substeps; /* collision on substeps with si % N == N-1 (cloth_jacobi.rs:703-704) */
    float thickness;                  /* THICKNESS (cloth_compute.rs:72) */
    float coll_scale;                 /* DEFAULT_COLL_SCALE (cloth_compute.rs:74) */
    float hash_cell;                  /* spatial hash cell edge [m], must be >= thickness */
    uint32_t hash_table_bits;         /* hash table of 2^bits buckets */
    uint32_t ring_depth;              /* for XPBD_COLLISION_RING_FILTER */
    uint32_t ground_enabled;
    float ground_y;
    uint32_t use_graphs;              /* capture each frame as a CUDA graph */
    float barrier_timeout_ms;         /* bound on every grid-barrier wait (default 2000) */
    uint32_t block_threads;           /* 0 = autotuned / default */
    uint32_t blocks_per_sm;           /* 0 = autotuned / default */
    uint32_t warm_start;              /* convergence solve start: XPBD_WARM_* (0 = plain, λ = 0) */
    uint32_t cluster_ctas;            /* Gauss–Seidel in one thread-block cluster: 0 auto, 1 off, 8 or 16 CTAs */
    uint32_t jacobi_kernel;           /* Jacobi: 0 default (= 5 where it applies, else 3), 1 warp tiles, 2 shared-
                                         memory patches (their tables are built by the first call that selects them,
                                         or by xpbd_autotune, which tries them for plain Jacobi), 3 thread per
                                         particle, 4 cloth-resident (each cloth in the shared memory of one CTA or a
                                         cluster of up to 16 for a whole frame, each constraint solved once per
                                         pass; λ cleared per pass, no collision, every cloth at most 65,536
                                         particles with particle-disjoint color batches — otherwise 3 runs),
                                         5 small batch (at most 8,192 particles: the whole batch in one cluster,
                                         thread per constraint record; the default up to 4,096 particles) */
    float tolerance;                  /* > 0 (or warm_start != 0): convergence solve — Jacobi, λ kept per substep,
                                         iterate until max |C + α̃λ|/rest <= tolerance, at most inner_iterations */
    uint32_t gs_strips;               /* Gauss–Seidel over several clusters: 0 / 1 none (xpbd_autotune may pick
                                         strips where they time faster), S >= 2 strips of
                                         cluster_ctas (16, or 8) CTAs each, particles shared between strips in
                                         global memory and ordered by per-CTA step flags (bounded waits) */
    uint32_t reserved[2];
} xpbd_solver_opts;

/* One cloth: the arrays of ClothMeshData / ClothSimConfig (mesh_prep.rs:103-131, cloth_compute.rs:140-179). All
 * host pointers; copied by xpbd_add_cloth. Optional arrays may be NULL. */
typedef struct xpbd_cloth_desc {
    uint32_t num_particles;
    const float* positions;           /* 3N, initial_pos */
    const float* velocities;          /* 3N or NULL (zero) */
    const float* inv_mass;            /* N, 0 = pinned */
    const float* rest_positions;      /* 3N or NULL (= positions); used by the collision rest filter */
    uint32_t num_constraints;
    const uint32_t* constraint_i;
    const uint32_t* constraint_j;
    const float* rest_len;
    const float* compliance;
    const uint32_t* constraint_type;  /* E or NULL (all stretch); XPBD_CONSTRAINT_* */
    uint32_t order;                   /* XPBD_ORDER_* */
    const uint32_t* batch_offsets;    /* XPBD_ORDER_PRESORTED only: batch_count+1 entries */
    uint32_t batch_count;
} xpbd_cloth_desc;

typedef struct xpbd_stats {
    uint64_t frames;
    uint64_t substeps;
    uint32_t num_particles;
    uint32_t num_constraints;
    uint32_t num_cloths;
    uint32_t num_colors;              /* max color batches over cloths (Gauss–Seidel sweep length) */
    uint32_t grid_blocks;
    uint32_t block_threads;
    uint32_t graph_captured;
    uint32_t cooperative_launch;
    uint64_t kernel_launches;         /* launches issued by the library so far (graph nodes count once each) */
    uint64_t warm_start_fallbacks;    /* substeps where the learned warm start was rejected */
    uint64_t collision_pairs;         /* pairs found by the last collision pass (when counted) */
    uint32_t solver_kernel;           /* 0 Jacobi warp tiles, 1 Gauss–Seidel grid, 2 Jacobi patches, 3 GS cluster,
                                         5 Jacobi thread per particle, 6 Jacobi convergence solve */
    uint32_t cluster_ctas;            /* CTAs of the Gauss–Seidel cluster (0 = grid kernel) */
    uint64_t converge_iterations;     /* convergence solve: update passes summed over substeps */
    uint64_t converge_substeps;
    uint32_t converge_max_iterations;
    uint32_t pad;
} xpbd_stats;

typedef struct xpbd_ctx xpbd_ctx;

/* ---- lifetime ---------------------------------------------------------------------------------------------- */
/* init_cloth_sim (cloth_compute.rs:571-623 → cloth_jacobi.rs:213-569): creates the context on `device`. */
int xpbd_create(xpbd_ctx** out, int device);
void xpbd_destroy(xpbd_ctx* ctx);
void xpbd_default_opts(xpbd_solver_opts* opts);
/* Use a caller stream (cudaStream_t as void*, NULL = the context's own stream). */
int xpbd_set_stream(xpbd_ctx* ctx, void* stream);

/* ---- building the batch ------------------------------------------------------------------------------------ */
/* ClothMeshData::to_sim_config + the buffer creation of init_cloth_sim_jacobi (cloth_compute.rs:1597-1705,
 * cloth_jacobi.rs:213-569, pack_neighbor_gpu :95-111). Cloths are packed by offset tables; ids count from 0. */
int xpbd_add_cloth(xpbd_ctx* ctx, const xpbd_cloth_desc* desc, uint32_t* cloth_id);
/* Builds coloring, neighbour tables and device buffers for every added cloth. */
int xpbd_commit(xpbd_ctx* ctx);
/* Kinematic grab of one vertex per cloth (extension of the single grab of xpbd_time_step_params, which stays): after
 * each prediction the cloth's local vertex `vertex` moves by stiffness·(target − x), at most 0.065 per substep
 * (xpbd_cpu.rs:56-63). vertex < 0 releases it. Takes effect from the next frame; no graph recapture. */
int xpbd_set_cloth_grab(xpbd_ctx* ctx, uint32_t cloth_id, int32_t vertex, const float* target_xyz, float stiffness);
/* Wind on one cloth (an extension; the reference has no wind): after gravity, the predicted velocity of every unpinned
 * particle of the cloth relaxes toward `velocity` (3 floats, m/s): v += (velocity - v) * (drag * dt). drag = 0 turns
 * it off (velocity may then be NULL). Takes effect from the next frame; no graph recapture. */
int xpbd_set_cloth_wind(xpbd_ctx* ctx, uint32_t cloth_id, const float* velocity, float drag);
/* Render triangles of a cloth (3 local vertex indices each; before xpbd_commit), for xpbd_read_normals. */
int xpbd_set_triangles(xpbd_ctx* ctx, uint32_t cloth_id, uint32_t num_tris, const uint32_t* tri_indices);
/* Vertex normals of the current positions, accumulate_normals + finalize_normals (cloth_sim_jacobi.wgsl:492-547):
 * area-weighted fixed-point sums (×33333, truncation) normalised, (0, 1, 0) where degenerate. xyz per vertex. */
int xpbd_read_normals(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz);

/* ---- per-frame --------------------------------------------------------------------------------------------- */
/* prepare_cloth_bind_groups_jacobi's per-frame ClothSimParamsGpu::pack upload (cloth_jacobi.rs:583-584). */
int xpbd_set_params(xpbd_ctx* ctx, const xpbd_time_step_params* params, const xpbd_solver_opts* opts);
/* run_cloth_sim_jacobi / run_cloth_sim_gauss_seidel (cloth_jacobi.rs:675-916, cloth_compute.rs:1271-1522):
 * enqueue `frames` frames of opts.substeps substeps each on the context stream (asynchronous). */
int xpbd_step(xpbd_ctx* ctx, uint32_t frames);
/* Headless `step(params)`: set_params(params, current opts) + step(frames). */
int xpbd_step_params(xpbd_ctx* ctx, const xpbd_time_step_params* params, uint32_t frames);
/* Enqueue single substeps (xpbd_substep_no_collision / _with_self_collision, xpbd_cpu.rs:411-578). */
int xpbd_substep(xpbd_ctx* ctx, uint32_t substeps);
/* Wait for the stream and report device-side errors. */
int xpbd_sync(xpbd_ctx* ctx);

/* ---- state ------------------------------------------------------------------------------------------------- */
/* Readback of sim_pos / velocities (gpu_cpu_parity_jacobi.rs:766-797). cloth_id = UINT32_MAX reads all. */
int xpbd_read_positions(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz);
int xpbd_read_velocities(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz);
int xpbd_write_state(xpbd_ctx* ctx, uint32_t cloth_id, const float* xyz, const float* vel_xyz);
/* reset_cloth_sim_state_jacobi (cloth_jacobi.rs:918-944): back to the initial positions, zero velocity and λ. */
int xpbd_reset(xpbd_ctx* ctx);
/* Per-constraint λ after the last substep, in the cloth's input constraint order (extension). */
int xpbd_read_lambda(xpbd_ctx* ctx, uint32_t cloth_id, float* out);
/* Convergence solve: the max pre-update residual max|C + α̃λ|/rest of each update pass of the most recent substep
 * (`count` = its number of passes; up to max_count values are copied). Extension: no reference counterpart. */
int xpbd_converge_history(xpbd_ctx* ctx, float* residuals, uint32_t max_count, uint32_t* count);
/* Convergence solve: update passes each cloth took in the most recent substep (out[num_cloths]). Extension. */
int xpbd_converge_cloth_iterations(xpbd_ctx* ctx, uint32_t* out);
/* Warm-start λ0 per constraint of a cloth (input order) for XPBD_WARM_GIVEN — extension. */
int xpbd_set_warm_lambda(xpbd_ctx* ctx, uint32_t cloth_id, const float* lambda0);
/* Max strain residual |‖xi−xj‖−rest|/rest over the constraints of a cloth (UINT32_MAX = all) — extension. */
int xpbd_strain_residual(xpbd_ctx* ctx, uint32_t cloth_id, float* out);
int xpbd_get_stats(xpbd_ctx* ctx, xpbd_stats* out);
/* Color batches of a cloth: perm[k] = input index of the k-th batch-sorted constraint; offsets has batch_count+1
 * entries (mesh_prep.rs:153-221). Pass NULL to query only *batch_count. */
int xpbd_get_coloring(xpbd_ctx* ctx, uint32_t cloth_id, uint32_t* perm, uint32_t* offsets, uint32_t* batch_count);

/* Host-only (no device needed): greedy edge coloring of one cloth's constraints exactly as
 * partition_constraints_for_gs_batches (mesh_prep.rs:153-221) — order XPBD_ORDER_COLOR_REFERENCE — or in plain index
 * order (XPBD_ORDER_COLOR_INDEX). perm: num_constraints entries; offsets: num_constraints+1 entries capacity. */
int xpbd_color_constraints(uint32_t num_particles, uint32_t num_constraints, const uint32_t* constraint_i,
                           const uint32_t* constraint_j, uint32_t order, uint32_t* perm, uint32_t* offsets,
                           uint32_t* batch_count);

/* ---- autotuning -------------------------------------------------------------------------------------------- */
/* Times `frames` frames per candidate schedule on a snapshot of the state, restores the state and keeps the fastest.
 * Candidates: Jacobi execution (spatial patches — their tables built here if needed —, thread per particle, warp
 * tiles) × block size × resident blocks per SM, plus the cloth-resident and small-batch kernels where they apply;
 * Gauss–Seidel: grid kernel × block × blocks per SM, clusters of 16 or 8 CTAs, and 2 / 4 / 8 strips of 16 CTAs. Writes the chosen block_threads / blocks_per_sm / cluster_ctas / jacobi_kernel / gs_strips to opts_out. */
int xpbd_autotune(xpbd_ctx* ctx, uint32_t frames, xpbd_solver_opts* opts_out);

/* ---- collision pipeline introspection (bit-exact parity tests) ---------------------------------------------- */
/* Runs the spatial hash on the current positions: keys[i] = hash(cell(x_i)) & (2^bits-1); then the stable LSD
 * radix sort (8-bit digits, one pass per 8 bits of the table; the same order as 4 passes) of (key, particle
 * index). Any output may be NULL. */
int xpbd_collision_keys(xpbd_ctx* ctx, uint32_t* keys, uint32_t* sorted_keys, uint32_t* sorted_vals);
/* Collision pairs (a<b, lexicographic) of the current positions under opts.collision; *count = total pairs,
 * at most `cap` written as (a,b) uint32 pairs. */
int xpbd_collision_pairs(xpbd_ctx* ctx, uint32_t* pairs, uint64_t cap, uint64_t* count);

/* ---- standalone device primitives (device pointers, caller stream) ----------------------------------------- */
/* Stable LSD radix sort of 32-bit keys with 32-bit payload, 8-bit digits, `passes` (1..4) passes from the least
 * significant digit. keys_in/vals_in are not modified. `scratch` must hold xpbd_radix_sort_scratch_bytes(n).
 * n may be at most XPBD_RADIX_SORT_MAX_KEYS (larger n: XPBD_ERR_CAPACITY, and a scratch size of 0). The two output
 * arrays must not overlap each other or either input array (XPBD_ERR_INVALID_ARGUMENT); the inputs may overlap. */
#define XPBD_RADIX_SORT_MAX_KEYS (1u << 31)
size_t xpbd_radix_sort_scratch_bytes(uint32_t n);
int xpbd_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out, uint32_t* vals_out,
                          uint32_t n, uint32_t passes, void* scratch, size_t scratch_bytes, void* stream);
/* The same sort for callers that cannot allocate device memory — e.g. code running where cudaMalloc is forbidden
 * or would stall (inside a frame budget where its implicit device synchronisation is not acceptable, under a host
 * application that reserves all device memory through its own pool, or in a plugin that may not grow the process's
 * footprint). No counterpart in the reference. It allocates nothing: its scratch is a fixed device array built into
 * the library, sized for at most XPBD_NOALLOC_SORT_MAX_KEYS keys (about 2.2 MB, held on every GPU that loads the
 * library until the process exits); larger n returns XPBD_ERR_CAPACITY. The array overlap rules are those of
 * xpbd_radix_sort_pairs. The first call on a device looks up the array's device address in the current context
 * (make it before any stream capture on that device); after the context is re-created (cudaDeviceReset), the next
 * call looks it up again. Every call shares the one array, so calls whose work overlaps on the GPU (other streams,
 * other host threads) race; serialise them. */
#define XPBD_NOALLOC_SORT_MAX_KEYS (1u << 18)
int xpbd_radix_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                  uint32_t* vals_out, uint32_t n, uint32_t passes, void* stream);
/* Greedy edge coloring on the GPU, bit-identical to the host coloring xpbd_color_constraints and so to
 * partition_constraints_for_gs_batches (mesh_prep.rs:153-221): the same colors, the same (color, index) batch order.
 * Device arrays: constraint_i/j[num_constraints]; perm[num_constraints] = input index of the k-th batch-sorted
 * constraint; colors[num_constraints] (may be NULL) = color of each input constraint; offsets[num_constraints + 2]
 * receives batch_count + 1 batch starts (no constraints: one empty batch, offsets {0, 0}). *batch_count is written on
 * the host, so the call synchronises `stream`; the rest of the work is enqueued on it.
 * A batch of cloths with disjoint particle ranges may be colored in one call: each cloth gets the coloring it would
 * get alone, and perm is then color-major across the cloths (the batch's Gauss–Seidel order). Give the cloths'
 * constraint ranges when they are known — cloth_constraint_offsets (host, num_cloths + 1 entries, from 0 to
 * num_constraints): each cloth is then colored by one thread block of its own, much faster than the schedule over
 * the whole grid used for num_cloths = 0 (one graph of unknown structure). Constraints of different cloths sharing a
 * particle: XPBD_ERR_INVALID_ARGUMENT. Endpoints out of range or i == j: XPBD_ERR_INDEX_RANGE. `scratch` (256-byte
 * aligned) must hold xpbd_color_constraints_device_scratch_bytes(num_particles, num_constraints, num_cloths) bytes
 * (about 56 bytes per constraint). */
size_t xpbd_color_constraints_device_scratch_bytes(uint32_t num_particles, uint32_t num_constraints,
                                                   uint32_t num_cloths);
int xpbd_color_constraints_device(uint32_t num_particles, uint32_t num_constraints, const uint32_t* constraint_i,
                                  const uint32_t* constraint_j, uint32_t order, uint32_t num_cloths,
                                  const uint32_t* cloth_constraint_offsets, uint32_t* perm, uint32_t* colors,
                                  uint32_t* offsets, uint32_t* batch_count, void* scratch, size_t scratch_bytes,
                                  void* stream);
/* Particle-major neighbour table of finalize_cloth_mesh (mesh_prep.rs:588-635) on the GPU, for constraints already in
 * batch order (device arrays): row_off[num_particles + 1]; row p of other/eid[2 * num_constraints] lists, in
 * increasing constraint position (i slot before j slot), the opposite endpoint and the constraint position of every
 * constraint at p. Synchronises `stream` once (index check). `scratch` (256-byte aligned) must hold
 * xpbd_neighbor_table_device_scratch_bytes(num_particles, num_constraints) bytes. */
size_t xpbd_neighbor_table_device_scratch_bytes(uint32_t num_particles, uint32_t num_constraints);
int xpbd_neighbor_table_device(uint32_t num_particles, uint32_t num_constraints, const uint32_t* constraint_i,
                               const uint32_t* constraint_j, uint32_t* row_off, uint32_t* other, uint32_t* eid,
                               void* scratch, size_t scratch_bytes, void* stream);
/* keys[i] = prime-hash(floor(xyz_i * inv_cell)) & (2^bits - 1), positions as float4 (w ignored). */
int xpbd_hash_keys(const float* xyzw, uint32_t n, float inv_cell, uint32_t table_bits, uint32_t* keys,
                   void* stream);

/* ---- learned warm start (extension: no reference counterpart) -------------------------------------------------
 * A 9→64→64→1 MLP (SiLU; BF16 tensor-core tiles, FP32 accumulation) predicting each constraint's initial λ for the
 * convergence solve (XPBD_WARM_LEARNED). Parameters: XPBD_MLP_PARAMS fp32 values in the order w1[64][9], b1[64],
 * w2[64][64], b2[64], w3[64], b3, plus XPBD_MLP_NORM normalisation values (feature mean[9], std[9], target mean,
 * std; features f0..f4 are standardised; the target is t = λ·(wi+wj+α̃)/rest and the network predicts its change over
 * the previous substep, t - f1, standardised with the target mean/std). */
#define XPBD_MLP_PARAMS 4865
#define XPBD_MLP_NORM 20
#define XPBD_MLP_FEATURES 9
/* Allocates the MLP (seeded initialisation) and a training set of `capacity` samples. */
int xpbd_mlp_init(xpbd_ctx* ctx, uint64_t seed, uint32_t capacity);
int xpbd_mlp_set_params(xpbd_ctx* ctx, const float* params, const float* norm);
int xpbd_mlp_get_params(xpbd_ctx* ctx, float* params, float* norm);
/* λ0 the learned warm start would give cloth `cloth`'s constraints (input order) at the next substep's predicted
 * positions; the simulation state is unchanged. */
int xpbd_mlp_predict_lambda(xpbd_ctx* ctx, uint32_t cloth, float* lambda0);
/* Runs `substeps` substeps of the convergence solve as configured (tolerance > 0; warm start, inner_iterations as set)
 * and stores, for every `stride`-th constraint (offset rotating per substep), its features at the substep's predicted
 * positions and its final λ as the target. */
int xpbd_mlp_collect(xpbd_ctx* ctx, uint32_t substeps, uint32_t stride);
int xpbd_mlp_dataset_size(xpbd_ctx* ctx, uint32_t* count);
/* Copies up to `max_rows` stored samples (raw features n x 9, targets t) to the host. */
int xpbd_mlp_dataset_read(xpbd_ctx* ctx, uint32_t max_rows, float* features, float* targets, uint32_t* rows);
/* Sets the standardisation from the stored samples. */
int xpbd_mlp_fit_normalization(xpbd_ctx* ctx);
/* `steps` Adam steps on minibatches of `batch` samples drawn (seeded) from the stored set; losses[steps] (may be NULL)
 * receives each step's mean squared error of the standardised target. */
int xpbd_mlp_train(xpbd_ctx* ctx, uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses);
/* Data-parallel training, one step in two calls so that the caller can sum the gradients over ranks in between (one
 * all-reduce of XPBD_MLP_PARAMS floats per step). Both run asynchronously on the context's stream; `grads` and `loss`
 * are device pointers. minibatch_gradients: gradient of the mean loss over `batch` stored samples drawn with `seed`
 * (xorshift64, as xpbd_mlp_train), written to grads[XPBD_MLP_PARAMS], the summed squared error to loss[0].
 * apply_gradients: one Adam step with the gradient grads·scale (scale = 1/ranks after a summing all-reduce). */
int xpbd_mlp_minibatch_gradients(xpbd_ctx* ctx, uint32_t batch, uint64_t seed, float* grads, float* loss);
int xpbd_mlp_apply_gradients(xpbd_ctx* ctx, const float* grads, float scale, float lr);
/* Standardised prediction for n raw feature rows (host arrays). */
int xpbd_mlp_eval(xpbd_ctx* ctx, const float* features, uint32_t n, float* out);
/* Gradient of mean((y - (t - f1 - tmean)/tstd)^2) over n rows w.r.t. the XPBD_MLP_PARAMS parameters (host arrays). */
int xpbd_mlp_gradients(xpbd_ctx* ctx, const float* features, const float* targets, uint32_t n, float* grads,
                       float* loss);

/* ---- cloth meshes: the crate's host-side mesh preparation (src/mesh_prep.rs) -------------------------------------
 * A built mesh holds positions, inverse masses (a third of 1/area of each incident triangle; top row pinned), render
 * triangles and its constraints — structural edges (α 2e-8), hinge bends (α 3.8), then the extras — already in the
 * greedy-colored batch order with batch offsets: pass them to xpbd_add_cloth with XPBD_ORDER_PRESORTED. */
typedef struct xpbd_mesh xpbd_mesh;
/* grid_cloth_hanging (mesh_prep.rs:363-406): quad grid in the XY plane, skip-2 braces and cross diagonals. */
int xpbd_mesh_grid_hanging(uint32_t quad_cols, uint32_t quad_rows, float cell_size, xpbd_mesh** out);
/* parse_welded_obj (mesh_prep.rs:223-357): vertices welded by corner string, quads split v0-v2 with a v1-v3 brace,
 * n-gons fanned, skip-2 braces when the vertices form an axis-aligned grid. */
int xpbd_mesh_from_obj(const char* obj_text, xpbd_mesh** out);
/* finalize_cloth_mesh (mesh_prep.rs:532-659) of a triangle mesh with extra constraints (i, j, rest, compliance). */
int xpbd_mesh_from_triangles(uint32_t num_vertices, const float* positions_xyz, uint32_t num_tris,
                             const uint32_t* tri_indices, uint32_t num_extra, const uint32_t* extra_i,
                             const uint32_t* extra_j, const float* extra_rest, const float* extra_comp,
                             xpbd_mesh** out);
int xpbd_mesh_sizes(const xpbd_mesh* mesh, uint32_t* num_vertices, uint32_t* num_tris, uint32_t* num_constraints,
                    uint32_t* num_batches);
/* Copies out any of: positions (xyz), inverse masses, triangles (3 per), constraint i/j/rest/compliance (batch
 * order), batch offsets (num_batches + 1). NULL skips an array. */
int xpbd_mesh_get(const xpbd_mesh* mesh, float* positions_xyz, float* inv_mass, uint32_t* tri_indices,
                  uint32_t* constraint_i, uint32_t* constraint_j, float* rest_len, float* compliance,
                  uint32_t* batch_offsets);
void xpbd_mesh_free(xpbd_mesh* mesh);

/* ---- diagnostics ------------------------------------------------------------------------------------------- */
const char* xpbd_last_error(xpbd_ctx* ctx);
const char* xpbd_status_string(int status);
/* Test hook for failure detection: the next step's first grid barrier expects one block more than the grid has,
 * so it can never complete and times out after `timeout_ms`, setting XPBD_ERR_BARRIER_TIMEOUT. */
int xpbd_debug_force_barrier_timeout(xpbd_ctx* ctx, float timeout_ms);
/* Self test of the kernels' shared-reciprocal division (three quotients from one correctly rounded reciprocal) against
 * the ordinary correctly rounded division on `count` random operand triples: *mismatches = differing quotients. */
int xpbd_selftest_division(int device, uint64_t count, uint64_t seed, uint64_t* mismatches);

#ifdef __cplusplus
}
#endif
#endif /* XPBD_CUDA_H */
