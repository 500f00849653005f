// Internal layout of the packed cloth batch in HBM, shared by the host runtime and the sm_100a kernels.
//
// All cloths of a context are packed back to back (vertex offsets, constraint offsets). Vertex state is float4
// per particle with w = inverse mass, so a neighbour gather brings position and mass in one 16-byte load:
//   x      sim positions            (reference sim_pos, vec4 w=0 in cloth_sim_jacobi.wgsl:27)
//   v      velocities               (w unused)
//   jac[2] Jacobi ping-pong buffers (reference jac_a / jac_b); jac[0] is the Gauss–Seidel working state
//   rest   rest positions           (collision rest filter)
// Jacobi neighbour table (CSR over particles, rows of pinned particles left empty):
//   row_off[n+1], inc[n_inc] = {other | palette<<28, rest bits}: 8 bytes per incidence. The compliance of an
//   incidence is palette_comp[cloth*16 + palette] (at most 16 distinct compliance values per cloth).
//   tiles[]: warp tiles of up to 32 consecutive particles of one cloth {first particle, count, cloth}.
// Gauss–Seidel constraints, color-major over the whole batch: con[e] = {i, j, rest bits, compliance bits},
//   color_off[ncolors+1]; λ per constraint in con_lambda.
#pragma once
#include <stdint.h>
#include <vector_types.h>

#define XPBD_PALETTE 16
#define XPBD_OTHER_MASK 0x0FFFFFFFu
#define XPBD_MAX_PARTICLES (1u << 28)

// Device status word values (mirror the negative XPBD_ERR_* codes as positive flags).
#define XPBD_DEV_NONFINITE 1
#define XPBD_DEV_BARRIER_TIMEOUT 2
#define XPBD_DEV_CAPACITY 4
#define XPBD_DEV_INDEX 8

struct XpbdDevParams {  // the per-call uniform block (ClothSimParamsGpu, cloth_compute.rs:245-273, + extensions)
    float dt, inv_dt, inv_dt_sq, omega;
    uint32_t iterations, relaxation, lambda_mode, solver;
    float gravity[3];
    float damp;  // exp(-linear_drag_per_sec * dt), evaluated on the host
    int32_t grab_idx;
    uint32_t grab_active;
    float grab_stiffness;
    float grab_target[3];
    float thickness, coll_scale, inv_cell, ground_y;
    uint32_t ground_enabled, collision, table_bits, warm_start;
    unsigned long long barrier_timeout_ns;
    float tolerance;       // convergence solve: stop when max |C + α̃λ|/rest of the pre-update state <= tolerance
    uint32_t max_iterations;
    // 1 when every α̃ = compliance·inv_dt_sq is finite and every free particle's inverse mass is >= 1e-8 (checked on
    // the host): then −C − α̃·0 is −C bit for bit and no constraint at a free particle has w sum < 1e-8, so the
    // reset-mode Jacobi term skips both evaluations
    uint32_t plain_terms;
};

#define XPBD_MLP_IN 9
#define XPBD_MLP_PARAMS 4865  // w1 64x9, b1 64, w2 64x64, b2 64, w3 64, b3 1 (fp32 master layout)
#define XPBD_MLP_NORM 20      // feature mean[9], std[9], target mean, std

// Working copy of the warm-start MLP read by the kernels: bf16 weights ([out][in], layer-1 inputs padded 9 → 16),
// fp32 biases, input/target standardisation.
struct XpbdMlp {
    uint16_t w1[64 * 16];
    uint16_t w2[64 * 64];
    uint16_t w3[64];
    float b1[64], b2[64], b3;
    float fmean[XPBD_MLP_IN], fstd[XPBD_MLP_IN], tmean, tstd;
};

#define XPBD_MAX_CONVERGE_ITERS 4096
struct XpbdConvergeStats {  // device counters of the convergence solve
    unsigned long long iterations;  // update passes summed over cloth-substeps
    unsigned long long substeps;    // cloth-substeps
    unsigned long long fallbacks;   // cloth-substeps whose warm start was rejected
    unsigned int max_iterations;
    unsigned int last_iterations;   // passes of the most recent substep, slowest cloth (its residuals stay in iter_res)
};

// Kinematic grab of one vertex of a cloth (the reference's mouse grab, one per cloth): after the prediction, the
// vertex is pulled toward the target by stiffness·(target − x), at most 0.065 per substep.
struct XpbdGrab {
    int32_t idx;  // global particle index, -1 = none
    float target[3];
    float stiffness;
    uint32_t pad[3];
};

// Wind on a cloth (extension, off by default): after gravity, every unpinned particle's predicted velocity relaxes
// toward the wind velocity, v += (wind - v) · (drag · dt).
struct XpbdWind {
    float vel[3];
    float drag;  // 1/s; 0 = no wind
};

struct XpbdGridSync {
    unsigned int count;
    unsigned int gen;
    unsigned int expected_extra;  // test hook: blocks the barrier expects beyond the grid (0 in normal runs)
    unsigned int pad;
};

struct XpbdTile {
    uint32_t first;  // first particle
    uint16_t count;  // particles in this tile (1..32)
    uint16_t cloth;  // cloth index (palette row)
};

// Spatial patch of the Jacobi solve: `np` owned particles (a recursive-coordinate-bisection block of one cloth) and
// `nh` halo particles read by its constraints. Local particle index: owned [0, np), halo [np, np+nh). All tables of
// a patch form one contiguous 16-byte aligned blob (fetched with one TMA bulk copy), sections 16-byte aligned:
//   parts[np+nh]   u32 global particle index (owned, then halo)
//   con[nc]        {li | lj<<12 | palette<<24, rest bits}: every constraint with an owned unpinned endpoint, solved
//                  once per patch per iteration
//   gofs[np+1]     per owned particle: range in `slots` of its incidences in neighbour-table order
//   slots[nslot]   u16 local constraint index | 0x8000 when the particle is the constraint's j endpoint
struct XpbdPatch {
    uint32_t off16;    // blob offset in 16-byte units
    uint32_t bytes;    // blob size (multiple of 16)
    uint32_t nc;       // constraints
    uint32_t lam_off;  // first λ slot of this patch's constraints
    uint16_t np, nh;
    uint16_t cloth, pad;
};
#define XPBD_PATCH_LOCAL_BITS 12
#define XPBD_PATCH_MAX_LOCAL (1u << XPBD_PATCH_LOCAL_BITS)
#define XPBD_PATCH_MAX_CON 32767u

// Cloth-resident Jacobi (jacobi_cloth_kernel): one CTA, or a cluster of `cl` CTAs, holds a whole cloth in shared
// memory for a frame. Rank r of the cluster owns the cloth-local particles [r·q, min(n, (r+1)·q)). A constraint
// endpoint is addressed as (rank << b) | local index, b = cloth_ep_bits(cl). Records are grouped by (color, rank): seg[seg_base + c·cl + r]
// is the first record of color c processed by rank r (the last entry closes the cloth's range).
struct XpbdClothDesc {
    uint32_t vtx_off;   // first particle of the cloth in the packed batch
    uint32_t n;         // particles
    uint32_t q;         // particles per rank (<= XPBD_CLOTH_RANK_MAX)
    uint32_t colors;    // color batches
    uint32_t seg_base;  // first entry of the cloth in seg[]
    uint32_t cl;        // CTAs of the cluster that solves the cloth
    uint32_t pad[2];
};
#define XPBD_CLOTH_EP_BITS 13          // local index bits of an endpoint for clusters of up to 8 CTAs
#define XPBD_CLOTH_RANK_MAX 7168u      // particles per CTA: 2 x 16 B of shared memory each (224 KB)
#define XPBD_CLOTH_MAX_CL 16u
// clusters of 16 CTAs (non-portable size) need four rank bits: 12 local bits, at most 4,096 particles per CTA
__host__ __device__ constexpr uint32_t cloth_ep_bits(uint32_t cl) { return cl > 8 ? 12u : 13u; }

struct XpbdWorld {  // device pointers + sizes, passed by value to kernels
    uint32_t n, e, n_inc, n_tiles, n_colors, n_cloths;
    float4* x;
    float4* v;
    float4* jac[2];
    float4* rest;
    const uint32_t* row_off;
    const uint2* inc;
    float* inc_lambda;
    const XpbdTile* tiles;
    const uint16_t* row_cloth;      // per particle: cloth index (palette row)
    const float* palette_comp;
    const float* inc_comp;          // per incidence compliance when a cloth has more than 16 values (else null)
    const uint4* con;
    float* con_lambda;
    const uint32_t* color_off;
    const uint4* con_in;            // constraints in input order, cloths contiguous (residual)
    const uint8_t* con_type;        // constraint type per packed input-order constraint
    const XpbdDevParams* params;
    int* status;
    XpbdGridSync* sync;
    // patch-staged Jacobi
    uint32_t n_patches, patch_max_local, patch_max_con, patch_con_total, patch_max_blob;
    const XpbdPatch* patches;
    const uint4* patch_blob;
    float* patch_lambda;
    // convergence solve
    float* warm_lam_inc;            // λ0 per incidence
    const uint32_t* inc_of_con;     // per constraint (input order, packed): incidence of the i / j side (2 entries)
    unsigned* cloth_res;            // 2 per cloth: plain / warm start residual (float bits)
    unsigned* iter_res;             // per iteration of a substep: residual of the still-active cloths (float bits)
    unsigned* cloth_ires;           // 3 x n_cloths: per-cloth residual of iterations it % 3 (float bits)
    unsigned* cloth_iters;          // per cloth: update passes of the current substep
    const XpbdGrab* grabs;          // per cloth
    const uint32_t* grab_count;     // number of cloths with an active grab (device word)
    const XpbdWind* winds;          // per cloth
    const uint32_t* wind_count;     // number of cloths with wind (device word)
    unsigned* div_exact;            // 3 slots: pass p of the row kernel takes the exact division when slot p % 3 != 0
    // render triangles (vertex normals)
    uint32_t n_tris;
    const uint4* tris;              // global vertex indices {a, b, c, 0}
    const uint32_t* vt_off;         // vertex → triangle table (CSR over vertices, triangles ascending)
    const uint32_t* vt_tri;
    float4* normals;
    XpbdConvergeStats* cstats;
};
