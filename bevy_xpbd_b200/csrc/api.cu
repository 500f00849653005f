// Host runtime behind include/xpbd_cuda.h: batch packing, device buffers, per-frame schedule, CUDA-graph capture,
// autotuning, state readback and device error reporting.
//
// Reference counterparts: init_cloth_sim_jacobi (buffer creation, cloth_jacobi.rs:213-569),
// prepare_cloth_bind_groups_jacobi (per-frame uniform upload, :571-649), run_cloth_sim_jacobi /
// run_cloth_sim_gauss_seidel (per-frame dispatch schedule, cloth_jacobi.rs:675-916, cloth_compute.rs:1271-1522),
// reset_cloth_sim_state_jacobi (:918-944).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <map>
#include <string>
#include <vector>
#include <thread>
#include <atomic>

#include "../../include/xpbd_cuda.h"
#include "mesh_prep.h"
#include "xpbd_internal.h"
#include "xpbd_kernels.h"

using namespace xpbd;

namespace {

struct ClothHost {
    uint32_t n = 0, e = 0;
    std::vector<float> pos, vel, w, rest_pos;
    std::vector<uint32_t> ci, cj, ctype;
    std::vector<float> rest, comp;
    uint32_t order = XPBD_ORDER_COLOR_REFERENCE;
    std::vector<uint32_t> given_offsets;
    // derived at commit
    std::vector<uint32_t> perm, colors, batch_off;
    uint32_t vtx_off = 0, con_off = 0;
    std::vector<uint32_t> lambda_inc;  // per input constraint: incidence holding its λ (Jacobi), or UINT32_MAX
    std::vector<uint32_t> lambda_gs;   // per input constraint: position in the color-major table
    std::vector<uint32_t> lambda_patch;  // per input constraint: patch slot holding its λ, or UINT32_MAX
    std::vector<uint32_t> inc_i, inc_j;  // per input constraint: incidence in the i / j particle's row (or MAX)
    std::vector<uint32_t> pal_idx;       // per input constraint: index of its compliance in the cloth's palette
    std::vector<uint32_t> tris;          // render triangles (local vertex indices), for the vertex normals
};

struct DeviceBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

}  // namespace

// bench.py counts this block as the per-step host→device bytes of the end-to-end path
static_assert(sizeof(XpbdDevParams) == 128, "update DEV_PARAMS_BYTES in bench.py");

struct xpbd_ctx {
    int device = 0;
    int sms = 148;
    bool coop_supported = false;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<ClothHost> cloths;
    bool committed = false;
    XpbdWorld W{};
    std::vector<void*> allocs;
    XpbdDevParams hp{};
    XpbdDevParams* dparams = nullptr;
    xpbd_time_step_params tsp{};
    xpbd_solver_opts opts{};
    bool params_set = false;
    CollisionBuffers cb{};
    bool coll_ready = false;
    uint32_t coll_ring_depth_built = 0;
    // schedule
    uint32_t block = 256, grid = 0;
    bool coop = false;
    uint32_t cl = 0;                 // >0: Gauss–Seidel runs in one cluster of `cl` CTAs
    uint32_t kernel = 0;             // solver kernel id (0 Jacobi tiles, 1 Gauss–Seidel, 2 Jacobi patches)
    bool patches_ok = false;         // patch tables built and usable (built on first use by ensure_patches)
    bool patches_tried = false;
    std::vector<uint4> con_host;     // color-major constraint table (host copy, for the cluster table)
    std::vector<uint32_t> color_off_host;
    ClusterTable ct{};
    uint32_t ct_cl = 0;
    // graph
    cudaGraphExec_t exec = nullptr;
    std::string graph_key;
    uint64_t graph_nodes = 0;
    // staging
    float* pinned = nullptr;
    size_t pinned_bytes = 0;
    float* d_xyz = nullptr;
    unsigned* d_resid = nullptr;
    int* d_status_copy = nullptr;
    xpbd_stats stats{};
    std::string last_error;
    // warm-start MLP
    XpbdMlp* d_mlp = nullptr;
    float *d_master = nullptr, *d_m1 = nullptr, *d_m2 = nullptr, *d_grads = nullptr, *d_loss = nullptr;
    float *d_feat = nullptr, *d_scale = nullptr, *d_target = nullptr;
    uint32_t* d_idx = nullptr;
    uint32_t idx_cap = 0, ds_count = 0, ds_cap = 0, collect_offset = 0;
    uint64_t adam_step = 0;
    float norm[XPBD_MLP_NORM] = {0};
    std::vector<XpbdGrab> grabs;  // per cloth (host copy)
    std::vector<XpbdWind> winds;  // per cloth (host copy)
    float forced_timeout_ms = 0.f;
    float w_min_free = INFINITY;  // smallest positive inverse mass of any cloth
    float comp_max = 0.f;         // largest compliance of any cloth
    // cloth-resident Jacobi (kernel id 7): per launch class the cloths it solves; side streams run the classes
    // concurrently (fork / join events on the context stream)
    bool wide_palette = false;       // a cloth has more than 16 compliance values: per-incidence compliances
    bool cloth_ok = false, cloth_tried = false;
    ClothSolveTable cloth_tab[kClothClasses] = {};
    cudaStream_t cls_stream[kClothClasses] = {};
    cudaEvent_t ev_fork = nullptr;
    cudaEvent_t ev_join[kClothClasses] = {};
    // Gauss–Seidel strips (kernel id 9)
    StripTable strip{};
    uint32_t strip_cl = 0, strip_s = 0, strip_block = 0;
    // single-cluster small batch (kernel id 8)
    bool small_ok = false, small_tried = false;
    SmallBatch small{};
    uint32_t small_cl = 0, small_block = 0;
};

// ------------------------------------------------------------------------------------------------- helpers
static int fail(xpbd_ctx* c, int code, const std::string& msg) {
    if (c) c->last_error = msg;
    return code;
}
static int cuda_fail(xpbd_ctx* c, cudaError_t e, const char* what) {
    int code = (e == cudaErrorMemoryAllocation) ? XPBD_ERR_OUT_OF_MEMORY : XPBD_ERR_CUDA;
    return fail(c, code, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t _e = (call);                         \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, what); \
    } while (0)

template <typename T>
static T* dev_alloc(xpbd_ctx* ctx, size_t count, cudaError_t* err) {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    *err = cudaMalloc(&p, bytes);
    if (*err == cudaSuccess) ctx->allocs.push_back(p);
    return (T*)p;
}

// Frees one buffer obtained from dev_alloc (growing scratch buffers replace theirs).
static void dev_release(xpbd_ctx* ctx, void* p) {
    if (!p) return;
    auto it = std::find(ctx->allocs.begin(), ctx->allocs.end(), p);
    if (it != ctx->allocs.end()) {
        ctx->allocs.erase(it);
        cudaFree(p);
    }
}

static void free_device(xpbd_ctx* ctx) {
    if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
    ctx->exec = nullptr;
    ctx->graph_key.clear();
    for (void* p : ctx->allocs) cudaFree(p);
    ctx->allocs.clear();
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
}

static void fill_dev_params(xpbd_ctx* ctx) {
    const xpbd_time_step_params& t = ctx->tsp;
    const xpbd_solver_opts& o = ctx->opts;
    XpbdDevParams& p = ctx->hp;
    p.dt = t.dt;
    p.inv_dt = t.inv_dt;
    p.inv_dt_sq = t.inv_dt * t.inv_dt;  // ClothSimParamsGpu::pack (cloth_compute.rs:325)
    p.omega = t.jacobi_omega;
    p.iterations = t.inner_iterations;
    p.relaxation = o.relaxation;
    p.lambda_mode = o.lambda_mode;
    p.solver = o.solver;
    for (int k = 0; k < 3; ++k) {
        p.gravity[k] = t.gravity[k];
        p.grab_target[k] = t.grab_target[k];
    }
    p.damp = expf(-t.linear_drag_per_sec * t.dt);  // xpbd_cpu.rs:402, one libm evaluation per upload
    p.grab_idx = t.grab_idx;
    p.grab_active = t.grab_active;
    p.grab_stiffness = t.grab_stiffness;
    p.thickness = o.thickness;
    p.coll_scale = o.coll_scale;
    p.inv_cell = 1.0f / std::max(o.hash_cell, o.thickness);
    p.ground_y = o.ground_y;
    p.ground_enabled = o.ground_enabled;
    p.collision = o.collision;
    p.table_bits = o.hash_table_bits;
    p.warm_start = o.warm_start;
    float tmo = ctx->forced_timeout_ms > 0.f ? ctx->forced_timeout_ms
                                             : (o.barrier_timeout_ms > 0.f ? o.barrier_timeout_ms : 2000.f);
    p.barrier_timeout_ns = (unsigned long long)((double)tmo * 1e6);
    p.tolerance = o.tolerance;
    p.max_iterations = t.inner_iterations;
    const float alpha_max = ctx->comp_max * p.inv_dt_sq;  // the largest α̃ any kernel forms (RN product, monotone)
    p.plain_terms = ctx->w_min_free >= 1e-8f && std::isfinite(p.inv_dt_sq) && std::isfinite(alpha_max) ? 1u : 0u;
    if (o.tolerance > 0.f || o.warm_start) p.lambda_mode = XPBD_LAMBDA_PER_SUBSTEP;
}

extern "C" void xpbd_default_opts(xpbd_solver_opts* o) {
    memset(o, 0, sizeof(*o));
    o->solver = XPBD_SOLVER_JACOBI;
    o->relaxation = XPBD_RELAX_OMEGA;
    o->lambda_mode = XPBD_LAMBDA_RESET_PER_ITERATION;
    o->substeps = 36;  // SUBSTEPS, cloth_compute.rs:59
    o->collision = XPBD_COLLISION_NONE;
    o->collision_every_n_substeps = 1;
    o->thickness = 0.04f;   // THICKNESS
    o->coll_scale = 0.38f;  // DEFAULT_COLL_SCALE
    o->hash_cell = 0.04f;
    o->hash_table_bits = 20;
    o->ring_depth = 2;
    o->use_graphs = 1;
    o->barrier_timeout_ms = 2000.f;
}

// ------------------------------------------------------------------------------------------------- lifetime
extern "C" int xpbd_create(xpbd_ctx** out, int device) {
    if (!out) return XPBD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return XPBD_ERR_NO_DEVICE;
    if (device < 0 || device >= count) return XPBD_ERR_INVALID_ARGUMENT;
    auto* ctx = new xpbd_ctx;
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, device);
    int coop = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete ctx;
        return XPBD_ERR_CUDA;
    }
    ctx->coop_supported = coop != 0;
    ctx->stream = ctx->own_stream;
    xpbd_default_opts(&ctx->opts);
    *out = ctx;
    return XPBD_OK;
}

extern "C" void xpbd_destroy(xpbd_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_device(ctx);
    for (int t = 0; t < kClothClasses; ++t) {
        if (ctx->cls_stream[t]) cudaStreamDestroy(ctx->cls_stream[t]);
        if (ctx->ev_join[t]) cudaEventDestroy(ctx->ev_join[t]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

extern "C" int xpbd_set_stream(xpbd_ctx* ctx, void* stream) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return XPBD_OK;
}

// ------------------------------------------------------------------------------------------------- building
extern "C" int xpbd_add_cloth(xpbd_ctx* ctx, const xpbd_cloth_desc* d, uint32_t* cloth_id) {
    if (!ctx || !d) return XPBD_ERR_INVALID_ARGUMENT;
    if (ctx->committed) return fail(ctx, XPBD_ERR_STATE, "xpbd_add_cloth after xpbd_commit");
    if (d->num_particles == 0 || !d->positions || !d->inv_mass)
        return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "cloth needs particles, positions and inv_mass");
    if (d->num_constraints > 0 && (!d->constraint_i || !d->constraint_j || !d->rest_len || !d->compliance))
        return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "constraint arrays missing");
    if (d->order > XPBD_ORDER_PRESORTED) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad constraint order mode");
    ClothHost c;
    c.n = d->num_particles;
    c.e = d->num_constraints;
    c.pos.assign(d->positions, d->positions + 3 * (size_t)c.n);
    c.vel.assign(3 * (size_t)c.n, 0.f);
    if (d->velocities) c.vel.assign(d->velocities, d->velocities + 3 * (size_t)c.n);
    c.w.assign(d->inv_mass, d->inv_mass + c.n);
    c.rest_pos = d->rest_positions ? std::vector<float>(d->rest_positions, d->rest_positions + 3 * (size_t)c.n)
                                   : c.pos;
    for (uint32_t i = 0; i < c.n; ++i) {
        if (!std::isfinite(c.w[i]) || c.w[i] < 0.f)
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "inv_mass must be finite and >= 0");
        for (int k = 0; k < 3; ++k)
            if (!std::isfinite(c.pos[3 * i + k])) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "non-finite position");
    }
    for (uint32_t i = 0; i < c.n; ++i)
        if (c.w[i] > 0.f) ctx->w_min_free = std::min(ctx->w_min_free, c.w[i]);
    if (c.e) {
        c.ci.assign(d->constraint_i, d->constraint_i + c.e);
        c.cj.assign(d->constraint_j, d->constraint_j + c.e);
        c.rest.assign(d->rest_len, d->rest_len + c.e);
        c.comp.assign(d->compliance, d->compliance + c.e);
        c.ctype.assign(c.e, XPBD_CONSTRAINT_STRETCH);
        if (d->constraint_type) c.ctype.assign(d->constraint_type, d->constraint_type + c.e);
        for (uint32_t e = 0; e < c.e; ++e) {
            if (c.ci[e] >= c.n || c.cj[e] >= c.n)
                return fail(ctx, XPBD_ERR_INDEX_RANGE, "constraint endpoint out of range");
            if (c.ci[e] == c.cj[e]) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "constraint joins a particle to itself");
            if (!(c.rest[e] >= 0.f) || !std::isfinite(c.rest[e]) || !(c.comp[e] >= 0.f) || !std::isfinite(c.comp[e]))
                return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "rest length / compliance must be finite and >= 0");
        }
        for (uint32_t e = 0; e < c.e; ++e) ctx->comp_max = std::max(ctx->comp_max, c.comp[e]);
    }
    c.order = d->order;
    if (d->order == XPBD_ORDER_PRESORTED) {
        if (!d->batch_offsets) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "presorted order needs batch_offsets");
        c.given_offsets.assign(d->batch_offsets, d->batch_offsets + d->batch_count + 1);
        if (c.given_offsets.front() != 0 || c.given_offsets.back() != c.e ||
            !std::is_sorted(c.given_offsets.begin(), c.given_offsets.end()))
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "batch_offsets must rise from 0 to num_constraints");
    }
    uint64_t total = (uint64_t)c.n;
    for (auto& o : ctx->cloths) total += o.n;
    if (total >= XPBD_MAX_PARTICLES) return fail(ctx, XPBD_ERR_CAPACITY, "more than 2^28 particles per context");
    if (ctx->cloths.size() >= 65535) return fail(ctx, XPBD_ERR_CAPACITY, "more than 65535 cloths per context");
    if (cloth_id) *cloth_id = (uint32_t)ctx->cloths.size();
    ctx->cloths.push_back(std::move(c));
    return XPBD_OK;
}

static void ensure_pinned(xpbd_ctx* ctx, size_t bytes) {
    if (ctx->pinned_bytes >= bytes) return;
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    if (cudaHostAlloc((void**)&ctx->pinned, bytes, cudaHostAllocDefault) == cudaSuccess) ctx->pinned_bytes = bytes;
}

extern "C" int xpbd_set_triangles(xpbd_ctx* ctx, uint32_t cloth_id, uint32_t num_tris, const uint32_t* tri_indices) {
    if (!ctx || (num_tris && !tri_indices)) return XPBD_ERR_INVALID_ARGUMENT;
    if (ctx->committed) return fail(ctx, XPBD_ERR_STATE, "xpbd_set_triangles after xpbd_commit");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    ClothHost& c = ctx->cloths[cloth_id];
    for (size_t k = 0; k < 3 * (size_t)num_tris; ++k)
        if (tri_indices[k] >= c.n) return fail(ctx, XPBD_ERR_INDEX_RANGE, "triangle vertex index out of range");
    c.tris.assign(tri_indices, tri_indices + 3 * (size_t)num_tris);
    return XPBD_OK;
}

// Runs fn(k) for k in [0, count) on up to hardware_concurrency host threads (each k exactly once).
template <typename Fn>
static void parallel_for(uint32_t count, Fn&& fn) {
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        for (uint32_t k = next++; k < count; k = next++) fn(k);
    };
    const uint32_t nthreads = std::max(1u, std::min<uint32_t>(count, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nthreads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
}

// XPBD_TRACE=1 in the environment: commit prints the host time of its phases to stderr.
static bool trace_enabled() {
    static const bool on = [] {
        const char* v = getenv("XPBD_TRACE");
        return v && *v && *v != '0';
    }();
    return on;
}

extern "C" int xpbd_commit(xpbd_ctx* ctx) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    auto t_last = std::chrono::steady_clock::now();
    auto mark = [&](const char* phase) {
        if (!trace_enabled()) return;
        const auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "[xpbd] commit %-28s %9.1f ms\n", phase,
                std::chrono::duration<double, std::milli>(now - t_last).count());
        t_last = now;
    };
    if (ctx->committed) return fail(ctx, XPBD_ERR_STATE, "already committed");
    if (ctx->cloths.empty()) return fail(ctx, XPBD_ERR_STATE, "no cloth added");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint32_t C = (uint32_t)ctx->cloths.size();
    uint32_t N = 0, E = 0, max_colors = 0;
    // ---- coloring (cloths are independent: one host thread per cloth at a time) + per-cloth offsets
    parallel_for(C, [&](uint32_t k) {
        ClothHost& c = ctx->cloths[k];
        if (c.order == XPBD_ORDER_PRESORTED) {
            c.perm.resize(c.e);
            for (uint32_t q = 0; q < c.e; ++q) c.perm[q] = q;
            c.batch_off = c.given_offsets;
            c.colors.assign(c.e, 0);
            for (size_t b = 0; b + 1 < c.batch_off.size(); ++b)
                for (uint32_t q = c.batch_off[b]; q < c.batch_off[b + 1]; ++q) c.colors[q] = (uint32_t)b;
        } else {
            color_constraints(c.n, c.e, c.ci.data(), c.cj.data(), c.order == XPBD_ORDER_COLOR_INDEX, c.perm, c.colors,
                              c.batch_off);
        }
    });
    for (auto& c : ctx->cloths) {
        c.vtx_off = N;
        c.con_off = E;
        N += c.n;
        E += c.e;
        max_colors = std::max<uint32_t>(max_colors, (uint32_t)c.batch_off.size() - 1);
    }
    mark("coloring");
    // ---- host tables: per cloth on parallel host threads (each writes only its own slices and its own local
    // tables), then concatenated in cloth order
    std::vector<float4> hx(N), hv(N), hrest(N);
    std::vector<uint32_t> row_off(N + 1, 0);
    std::vector<uint2> inc;
    std::vector<XpbdTile> tiles;
    std::vector<float> palette((size_t)C * XPBD_PALETTE, 0.f);
    std::vector<uint4> con_in(E);
    struct ClothTables {
        std::vector<uint2> inc;         // this cloth's incidences (rows in particle order)
        std::vector<float> inc_comp;    // their compliances (only when some cloth has more than 16 values)
        std::vector<uint32_t> row_off;  // local row starts (n)
        bool palette_ok = true;
    };
    std::vector<ClothTables> ct(C);
    // compliance palettes: up to 16 distinct values per cloth are named by 4 bits of the incidence record; a cloth
    // with more makes the whole batch carry a per-incidence compliance array instead
    parallel_for(C, [&](uint32_t ci_) {
        ClothHost& c = ctx->cloths[ci_];
        std::vector<float> pal;
        std::vector<uint32_t>& pidx = c.pal_idx;
        pidx.assign(c.e, 0);
        for (uint32_t e = 0; e < c.e; ++e) {
            uint32_t bits;
            memcpy(&bits, &c.comp[e], 4);
            size_t k = 0;
            for (; k < pal.size(); ++k) {
                uint32_t pb;
                memcpy(&pb, &pal[k], 4);
                if (pb == bits) break;
            }
            if (k == pal.size()) {
                if (pal.size() == XPBD_PALETTE) {
                    ct[ci_].palette_ok = false;
                    pidx.assign(c.e, 0);
                    return;
                }
                pal.push_back(c.comp[e]);
            }
            pidx[e] = (uint32_t)k;
        }
        for (size_t k = 0; k < pal.size(); ++k) palette[(size_t)ci_ * XPBD_PALETTE + k] = pal[k];
    });
    bool wide = false;
    for (uint32_t ci_ = 0; ci_ < C; ++ci_) wide = wide || !ct[ci_].palette_ok;
    ctx->wide_palette = wide;
    parallel_for(C, [&](uint32_t ci_) {
        ClothHost& c = ctx->cloths[ci_];
        ClothTables& t = ct[ci_];
        for (uint32_t i = 0; i < c.n; ++i) {
            hx[c.vtx_off + i] = make_float4(c.pos[3 * i], c.pos[3 * i + 1], c.pos[3 * i + 2], c.w[i]);
            hv[c.vtx_off + i] = make_float4(c.vel[3 * i], c.vel[3 * i + 1], c.vel[3 * i + 2], 0.f);
            hrest[c.vtx_off + i] =
                make_float4(c.rest_pos[3 * i], c.rest_pos[3 * i + 1], c.rest_pos[3 * i + 2], 0.f);
        }
        const std::vector<uint32_t>& pidx = c.pal_idx;
        // batch-sorted constraints and the neighbour table in reference order
        std::vector<uint32_t> si(c.e), sj(c.e);
        for (uint32_t k = 0; k < c.e; ++k) {
            si[k] = c.ci[c.perm[k]];
            sj[k] = c.cj[c.perm[k]];
        }
        std::vector<uint32_t> roff, other, eid;
        neighbor_csr(c.n, c.e, si.data(), sj.data(), roff, other, eid);
        c.lambda_inc.assign(c.e, 0xFFFFFFFFu);
        c.inc_i.assign(c.e, 0xFFFFFFFFu);
        c.inc_j.assign(c.e, 0xFFFFFFFFu);
        t.row_off.resize(c.n);
        t.inc.reserve(roff[c.n]);
        for (uint32_t i = 0; i < c.n; ++i) {
            t.row_off[i] = (uint32_t)t.inc.size();
            if (c.w[i] <= 0.f) continue;  // pinned rows stay empty: jacobi_gather returns jac_in for them
            for (uint32_t k = roff[i]; k < roff[i + 1]; ++k) {
                const uint32_t e_in = c.perm[eid[k]];
                uint32_t rb;
                memcpy(&rb, &c.rest[e_in], 4);
                if (c.lambda_inc[e_in] == 0xFFFFFFFFu) c.lambda_inc[e_in] = (uint32_t)t.inc.size();
                (c.ci[e_in] == i ? c.inc_i : c.inc_j)[e_in] = (uint32_t)t.inc.size();
                t.inc.push_back(make_uint2((other[k] + c.vtx_off) | (pidx[e_in] << 28), rb));
                if (wide) t.inc_comp.push_back(c.comp[e_in]);
            }
        }
        for (uint32_t e = 0; e < c.e; ++e) {
            uint32_t rb, cb;
            memcpy(&rb, &c.rest[e], 4);
            memcpy(&cb, &c.comp[e], 4);
            con_in[c.con_off + e] = make_uint4(c.ci[e] + c.vtx_off, c.cj[e] + c.vtx_off, rb, cb);
        }
    });
    // cloth k's incidences start at the total of the cloths before it; each cloth copies and rebases its own slice
    std::vector<size_t> inc_base(C + 1, 0);
    for (uint32_t ci_ = 0; ci_ < C; ++ci_) inc_base[ci_ + 1] = inc_base[ci_] + ct[ci_].inc.size();
    inc.resize(inc_base[C]);
    std::vector<float> inc_comp(wide ? inc_base[C] : 0);
    parallel_for(C, [&](uint32_t ci_) {
        ClothHost& c = ctx->cloths[ci_];
        ClothTables& t = ct[ci_];
        const uint32_t base = (uint32_t)inc_base[ci_];
        if (wide) std::copy(t.inc_comp.begin(), t.inc_comp.end(), inc_comp.begin() + base);
        for (uint32_t i = 0; i < c.n; ++i) row_off[c.vtx_off + i] = base + t.row_off[i];
        for (uint32_t e = 0; e < c.e; ++e) {
            if (c.lambda_inc[e] != 0xFFFFFFFFu) c.lambda_inc[e] += base;
            if (c.inc_i[e] != 0xFFFFFFFFu) c.inc_i[e] += base;
            if (c.inc_j[e] != 0xFFFFFFFFu) c.inc_j[e] += base;
        }
        std::copy(t.inc.begin(), t.inc.end(), inc.begin() + base);
        std::vector<uint2>().swap(t.inc);
        c.lambda_patch.assign(c.e, 0xFFFFFFFFu);
    });
    for (uint32_t ci_ = 0; ci_ < C; ++ci_) {
        const ClothHost& c = ctx->cloths[ci_];
        for (uint32_t first = 0; first < c.n; first += 32) {
            XpbdTile tile;
            tile.first = c.vtx_off + first;
            tile.count = (uint16_t)std::min<uint32_t>(32, c.n - first);
            tile.cloth = (uint16_t)ci_;
            tiles.push_back(tile);
        }
    }
    row_off[N] = (uint32_t)inc.size();
    mark("neighbour tables");
    // ---- Gauss–Seidel table, color-major across cloths: segment (color, cloth) starts after every earlier color
    // and, within its color, after the earlier cloths; each cloth fills its own segments
    std::vector<uint4> con(E);
    std::vector<uint32_t> color_off(max_colors + 1, 0);
    {
        std::vector<uint32_t> seg((size_t)max_colors * C + 1, 0);
        for (uint32_t col = 0; col < max_colors; ++col)
            for (uint32_t k = 0; k < C; ++k) {
                const ClothHost& c = ctx->cloths[k];
                const uint32_t cnt = col + 1 < c.batch_off.size() ? c.batch_off[col + 1] - c.batch_off[col] : 0u;
                seg[(size_t)col * C + k + 1] = seg[(size_t)col * C + k] + cnt;
            }
        for (uint32_t col = 0; col < max_colors; ++col) color_off[col] = seg[(size_t)col * C];
        color_off[max_colors] = seg[(size_t)max_colors * C];
        parallel_for(C, [&](uint32_t k) {
            ClothHost& c = ctx->cloths[k];
            if (c.lambda_gs.empty()) c.lambda_gs.assign(c.e, 0);
            for (uint32_t col = 0; col + 1 < c.batch_off.size() && col < max_colors; ++col) {
                uint32_t pos = seg[(size_t)col * C + k];
                for (uint32_t q = c.batch_off[col]; q < c.batch_off[col + 1]; ++q) {
                    const uint32_t e_in = c.perm[q];
                    con[pos] = con_in[c.con_off + e_in];
                    c.lambda_gs[e_in] = pos;
                    ++pos;
                }
            }
        });
    }
    mark("Gauss-Seidel table");
    // ---- device buffers
    cudaError_t err = cudaSuccess;
    XpbdWorld& W = ctx->W;
    W.n = N;
    W.e = E;
    W.n_inc = (uint32_t)inc.size();
    W.n_tiles = (uint32_t)tiles.size();
    W.n_colors = max_colors;
    W.n_cloths = C;
#define ALLOC(ptr, T, count)                                                         \
    do {                                                                             \
        ptr = dev_alloc<T>(ctx, (count), &err);                                      \
        if (err != cudaSuccess) { free_device(ctx); return cuda_fail(ctx, err, "cudaMalloc"); } \
    } while (0)
    float4 *x, *v, *j0, *j1, *rest;
    uint32_t *roff_d, *color_d;
    uint2* inc_d;
    float *lam_inc, *pal_d, *lam_con;
    XpbdTile* tiles_d;
    uint4 *con_d, *con_in_d;
    int* status;
    XpbdGridSync* sync;
    ALLOC(x, float4, N);
    ALLOC(v, float4, N);
    ALLOC(j0, float4, N);
    ALLOC(j1, float4, N);
    ALLOC(rest, float4, N);
    ALLOC(roff_d, uint32_t, N + 1);
    ALLOC(inc_d, uint2, inc.size());
    ALLOC(lam_inc, float, inc.size());
    float* inc_comp_d = nullptr;
    if (wide) ALLOC(inc_comp_d, float, inc.size());
    ALLOC(tiles_d, XpbdTile, tiles.size());
    uint16_t* rcloth_d;
    ALLOC(rcloth_d, uint16_t, N);
    ALLOC(pal_d, float, palette.size());
    ALLOC(con_d, uint4, E);
    ALLOC(lam_con, float, E);
    ALLOC(color_d, uint32_t, max_colors + 1);
    ALLOC(con_in_d, uint4, E);
    uint8_t* con_type_d;
    ALLOC(con_type_d, uint8_t, E);
    ALLOC(ctx->dparams, XpbdDevParams, 1);
    ALLOC(status, int, 4);
    ALLOC(sync, XpbdGridSync, 1);
    ALLOC(ctx->d_xyz, float, 3 * (size_t)N);
    float* warm_inc;
    uint32_t* inc_of_con_d;
    unsigned *cloth_res_d, *iter_res_d, *cloth_ires_d, *cloth_iters_d;
    XpbdConvergeStats* cstats_d;
    ALLOC(warm_inc, float, inc.size());
    ALLOC(inc_of_con_d, uint32_t, 2 * (size_t)E);
    ALLOC(cloth_res_d, unsigned, 2 * (size_t)C);
    ALLOC(iter_res_d, unsigned, XPBD_MAX_CONVERGE_ITERS);
    ALLOC(cloth_ires_d, unsigned, 3 * (size_t)C);
    ALLOC(cloth_iters_d, unsigned, C);
    ALLOC(cstats_d, XpbdConvergeStats, 1);
    ALLOC(ctx->d_resid, unsigned, 4);
    unsigned* div_exact_d;
    ALLOC(div_exact_d, unsigned, 4);
    XpbdGrab* grabs_d;
    uint32_t* grab_count_d;
    ALLOC(grabs_d, XpbdGrab, C);
    ALLOC(grab_count_d, uint32_t, 1);
    XpbdWind* winds_d;
    uint32_t* wind_count_d;
    ALLOC(winds_d, XpbdWind, C);
    ALLOC(wind_count_d, uint32_t, 1);
    ctx->winds.assign(C, XpbdWind{{0.f, 0.f, 0.f}, 0.f});
    ctx->grabs.assign(C, XpbdGrab{-1, {0.f, 0.f, 0.f}, 0.f, {0u, 0u, 0u}});
    // render triangles: packed global vertex indices and the vertex → triangle table for the vertex normals
    std::vector<uint4> tri_all;
    for (auto& c : ctx->cloths)
        for (size_t t = 0; t + 2 < c.tris.size(); t += 3)
            tri_all.push_back(make_uint4(c.tris[t] + c.vtx_off, c.tris[t + 1] + c.vtx_off, c.tris[t + 2] + c.vtx_off, 0u));
    const uint32_t T = (uint32_t)tri_all.size();
    std::vector<uint32_t> vt_off(N + 1, 0), vt_tri(3 * (size_t)T);
    for (const uint4& t : tri_all) {
        ++vt_off[t.x + 1];
        ++vt_off[t.y + 1];
        ++vt_off[t.z + 1];
    }
    for (uint32_t v = 0; v < N; ++v) vt_off[v + 1] += vt_off[v];
    {
        std::vector<uint32_t> cur(vt_off.begin(), vt_off.end() - 1);
        for (uint32_t t = 0; t < T; ++t) {
            vt_tri[cur[tri_all[t].x]++] = t;
            vt_tri[cur[tri_all[t].y]++] = t;
            vt_tri[cur[tri_all[t].z]++] = t;
        }
    }
    uint4* tris_d = nullptr;
    uint32_t *vt_off_d = nullptr, *vt_tri_d = nullptr;
    float4* normals_d = nullptr;
    if (T) {
        ALLOC(tris_d, uint4, T);
        ALLOC(vt_off_d, uint32_t, N + 1);
        ALLOC(vt_tri_d, uint32_t, 3 * (size_t)T);
        ALLOC(normals_d, float4, N);
    }
    cudaStream_t st = ctx->stream;
#define H2D(dst, src, bytes) CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st), "upload")
    H2D(x, hx.data(), N * sizeof(float4));
    H2D(v, hv.data(), N * sizeof(float4));
    H2D(j0, hx.data(), N * sizeof(float4));
    H2D(j1, hx.data(), N * sizeof(float4));
    H2D(rest, hrest.data(), N * sizeof(float4));
    H2D(roff_d, row_off.data(), (N + 1) * sizeof(uint32_t));
    if (!inc.empty()) H2D(inc_d, inc.data(), inc.size() * sizeof(uint2));
    if (wide && !inc.empty()) {
        H2D(inc_comp_d, inc_comp.data(), inc.size() * sizeof(float));
        CK(cudaStreamSynchronize(st), "commit sync");
    }
    CK(cudaMemsetAsync(lam_inc, 0, std::max<size_t>(inc.size(), 1) * sizeof(float), st), "memset");
    H2D(tiles_d, tiles.data(), tiles.size() * sizeof(XpbdTile));
    {
        std::vector<uint16_t> rc(N);
        parallel_for(C, [&](uint32_t k) {
            for (uint32_t i = 0; i < ctx->cloths[k].n; ++i) rc[ctx->cloths[k].vtx_off + i] = (uint16_t)k;
        });
        H2D(rcloth_d, rc.data(), N * sizeof(uint16_t));
        CK(cudaStreamSynchronize(st), "commit sync");
    }
    H2D(pal_d, palette.data(), palette.size() * sizeof(float));
    std::vector<uint8_t> ctypes(E);
    parallel_for(C, [&](uint32_t k) {
        const ClothHost& c = ctx->cloths[k];
        for (uint32_t e = 0; e < c.e; ++e) ctypes[c.con_off + e] = (uint8_t)std::min<uint32_t>(c.ctype[e], 2);
    });
    if (E) {
        H2D(con_d, con.data(), E * sizeof(uint4));
        H2D(con_in_d, con_in.data(), E * sizeof(uint4));
        H2D(con_type_d, ctypes.data(), E);
        CK(cudaStreamSynchronize(st), "commit sync");
    }
    CK(cudaMemsetAsync(lam_con, 0, std::max<size_t>(E, 1) * sizeof(float), st), "memset");
    H2D(color_d, color_off.data(), color_off.size() * sizeof(uint32_t));
    ctx->con_host = con;
    ctx->color_off_host = color_off;
    CK(cudaMemsetAsync(status, 0, 4 * sizeof(int), st), "memset");
    CK(cudaMemsetAsync(warm_inc, 0, std::max<size_t>(inc.size(), 1) * 4, st), "memset");
    CK(cudaMemsetAsync(cstats_d, 0, sizeof(XpbdConvergeStats), st), "memset");
    {
        std::vector<uint32_t> ioc(2 * (size_t)E);
        parallel_for(C, [&](uint32_t k) {
            const ClothHost& c = ctx->cloths[k];
            for (uint32_t e = 0; e < c.e; ++e) {
                ioc[2 * ((size_t)c.con_off + e)] = c.inc_i[e];
                ioc[2 * ((size_t)c.con_off + e) + 1] = c.inc_j[e];
            }
        });
        if (E) H2D(inc_of_con_d, ioc.data(), ioc.size() * 4);
        CK(cudaStreamSynchronize(st), "commit sync");
    }
    ctx->patches_ok = false;  // the spatial-patch tables are built on first use (ensure_patches)
    ctx->patches_tried = false;
    CK(cudaMemsetAsync(sync, 0, sizeof(XpbdGridSync), st), "memset");
    CK(cudaStreamSynchronize(st), "commit sync");
    W.x = x;
    W.v = v;
    W.jac[0] = j0;
    W.jac[1] = j1;
    W.rest = rest;
    W.row_off = roff_d;
    W.inc = inc_d;
    W.inc_lambda = lam_inc;
    W.tiles = tiles_d;
    W.row_cloth = rcloth_d;
    W.palette_comp = pal_d;
    W.inc_comp = inc_comp_d;
    W.con = con_d;
    W.con_lambda = lam_con;
    W.color_off = color_d;
    W.con_in = con_in_d;
    W.con_type = con_type_d;
    W.params = ctx->dparams;
    W.status = status;
    W.sync = sync;
    W.warm_lam_inc = warm_inc;
    W.inc_of_con = inc_of_con_d;
    W.cloth_res = cloth_res_d;
    W.iter_res = iter_res_d;
    W.cloth_ires = cloth_ires_d;
    W.cloth_iters = cloth_iters_d;
    W.div_exact = div_exact_d;
    W.grabs = grabs_d;
    W.grab_count = grab_count_d;
    H2D(grabs_d, ctx->grabs.data(), C * sizeof(XpbdGrab));
    CK(cudaMemsetAsync(grab_count_d, 0, sizeof(uint32_t), st), "memset");
    W.winds = winds_d;
    W.wind_count = wind_count_d;
    H2D(winds_d, ctx->winds.data(), C * sizeof(XpbdWind));
    CK(cudaMemsetAsync(wind_count_d, 0, sizeof(uint32_t), st), "memset");
    CK(cudaStreamSynchronize(st), "commit sync");
    CK(cudaMemsetAsync(div_exact_d, 0xFF, 4 * sizeof(unsigned), st), "memset");  // exact until the first check
    W.n_tris = T;
    W.tris = tris_d;
    W.vt_off = vt_off_d;
    W.vt_tri = vt_tri_d;
    W.normals = normals_d;
    if (T) {
        H2D(tris_d, tri_all.data(), T * sizeof(uint4));
        H2D(vt_off_d, vt_off.data(), (N + 1) * sizeof(uint32_t));
        H2D(vt_tri_d, vt_tri.data(), 3 * (size_t)T * sizeof(uint32_t));
        CK(cudaStreamSynchronize(st), "commit sync");
    }
    W.cstats = cstats_d;
    ensure_pinned(ctx, 16 * (size_t)N);
    mark("device buffers, uploads");
    ctx->committed = true;
    ctx->stats.num_particles = N;
    ctx->stats.num_constraints = E;
    ctx->stats.num_cloths = C;
    ctx->stats.num_colors = max_colors;
    return XPBD_OK;
}

// ------------------------------------------------------------------------------------------------- schedule
static uint32_t ceil_log2(uint32_t v) {
    uint32_t s = 0;
    while ((1u << s) < v) ++s;
    return s;
}

// Reorders rec[lo, hi) into runs of eight records (the eight lanes of one phase of a warp's 16-byte shared-memory
// access) whose two shared-memory slots lie in different 16-byte bank groups, as far as the remaining records allow:
// `banks(r)` names a record's class (first slot mod 8) · 8 + (second slot mod 8); each run takes, from the classes
// with the most records left first, those whose banks are still free in the run, then fills up with any.
template <typename Banks>
static void deal_bank_runs(std::vector<uint4>& rec, size_t lo, size_t hi, Banks banks) {
    std::vector<uint4> bucket[64];
    for (size_t k = lo; k < hi; ++k) bucket[banks(rec[k])].push_back(rec[k]);
    size_t next[64] = {};
    uint32_t byrem[64];
    for (size_t k = lo; k < hi;) {
        for (uint32_t q = 0; q < 64; ++q) byrem[q] = q;
        std::sort(byrem, byrem + 64, [&](uint32_t a, uint32_t b) {
            return bucket[a].size() - next[a] > bucket[b].size() - next[b];
        });
        uint32_t used_i = 0, used_j = 0, taken = 0;
        for (int pass = 0; pass < 2 && taken < 8 && k < hi; ++pass)
            for (uint32_t t = 0; t < 64 && taken < 8 && k < hi; ++t) {
                const uint32_t q = byrem[t], bi = q >> 3, bj = q & 7u;
                if (next[q] == bucket[q].size()) continue;
                if (pass == 0 && (((used_i >> bi) & 1u) || ((used_j >> bj) & 1u))) continue;
                used_i |= 1u << bi;
                used_j |= 1u << bj;
                rec[k++] = bucket[q][next[q]++];
                ++taken;
            }
    }
}

// Groups the color-major constraint table by (color, rank owning the first endpoint) for a cluster of `cl` CTAs.
static bool build_cluster_table(xpbd_ctx* ctx, uint32_t cl) {
    if (ctx->ct_cl == cl) return true;
    const uint32_t N = ctx->W.n;
    const uint32_t shift = ceil_log2((N + cl - 1) / cl);
    const uint32_t ncol = ctx->W.n_colors;
    std::vector<uint32_t> cnt((size_t)ncol * cl + 1, 0);
    for (uint32_t c = 0; c < ncol; ++c)
        for (uint32_t e = ctx->color_off_host[c]; e < ctx->color_off_host[c + 1]; ++e)
            ++cnt[(size_t)c * cl + (ctx->con_host[e].x >> shift) + 1];
    uint32_t max_chunk = 0;
    for (size_t k = 1; k < cnt.size(); ++k) max_chunk = std::max(max_chunk, cnt[k]);
    for (size_t k = 1; k < cnt.size(); ++k) cnt[k] += cnt[k - 1];
    if (cluster_gs_smem_bytes(shift, max_chunk) > 220 * 1024) return false;
    // boundary particles: endpoints of a constraint between two CTAs' particles (any color). Within each
    // (color, rank) group the records touching a boundary particle come first; the kernel solves them, signals the
    // cluster barrier, then solves the rest (only this CTA's interior particles) while the barrier completes.
    std::vector<uint8_t> bnd(N, 0);
    for (uint32_t e = 0; e < ctx->W.e; ++e) {
        const uint4 r = ctx->con_host[e];
        if ((r.x >> shift) != (r.y >> shift)) bnd[r.x] = bnd[r.y] = 1;
    }
    std::vector<uint4> rec(ctx->W.e);
    std::vector<uint32_t> nbd((size_t)ncol * cl, 0);
    std::vector<uint32_t> cur(cnt.begin(), cnt.end() - 1);
    for (int pass = 0; pass < 2; ++pass)  // boundary records, then interior records (bank-dealt below)
        for (uint32_t c = 0; c < ncol; ++c)
            for (uint32_t e = ctx->color_off_host[c]; e < ctx->color_off_host[c + 1]; ++e) {
                const uint4 r = ctx->con_host[e];
                const bool b = bnd[r.x] || bnd[r.y];
                if (b != (pass == 0)) continue;
                const size_t g = (size_t)c * cl + (r.x >> shift);
                rec[cur[g]++] = r;
                if (b) ++nbd[g];
            }
    // Within the boundary and the interior part of every group, the records are dealt in bank-spread runs of eight
    // (deal_bank_runs). A color's records share no particle, so their order within the color leaves every result
    // bit unchanged.
    const uint32_t lmask = (1u << shift) - 1u;
    for (uint4& r : rec) {  // endpoints as the kernel addresses them: rank << shift | shared-memory slot
        r.x = (r.x & ~lmask) | cluster_slot(r.x & lmask);
        r.y = (r.y & ~lmask) | cluster_slot(r.y & lmask);
    }
    auto gs_banks = [](const uint4& r) { return (r.x & 7u) * 8u + (r.y & 7u); };
    for (size_t g = 0; g + 1 < cnt.size(); ++g) {
        deal_bank_runs(rec, cnt[g], cnt[g] + nbd[g], gs_banks);
        deal_bank_runs(rec, cnt[g] + nbd[g], cnt[g + 1], gs_banks);
    }
    cudaError_t err = cudaSuccess;
    uint4* drec = dev_alloc<uint4>(ctx, rec.size(), &err);
    uint32_t *doff = nullptr, *dnbd = nullptr;
    if (err == cudaSuccess) doff = dev_alloc<uint32_t>(ctx, cnt.size(), &err);
    if (err == cudaSuccess) dnbd = dev_alloc<uint32_t>(ctx, nbd.size(), &err);
    if (err != cudaSuccess) return false;
    if (!rec.empty() && cudaMemcpy(drec, rec.data(), rec.size() * 16, cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    if (cudaMemcpy(doff, cnt.data(), cnt.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) return false;
    if (cudaMemcpy(dnbd, nbd.data(), nbd.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) return false;
    ctx->ct.rec = drec;
    ctx->ct.off = doff;
    ctx->ct.nbd = dnbd;
    ctx->ct.shift = shift;
    ctx->ct.max_chunk = std::max<uint32_t>(max_chunk, 1);
    ctx->ct_cl = cl;
    return true;
}

// Spatial patches for the shared-memory Jacobi kernel (jacobi_kernel 2), built on first use rather than in
// xpbd_commit: only that kernel reads them, and for large batches they are the costliest host table. Per cloth on
// parallel host threads, then concatenated in cloth order into one contiguous 16-byte aligned blob per patch
// (parts | con | gofs (patch-relative) | slots). Returns false when a cloth cannot be split into patches (the
// schedule then keeps the thread-per-particle kernel); allocation failures are errors.
static int ensure_patches(xpbd_ctx* ctx, bool* usable) {
    *usable = ctx->patches_ok;
    if (ctx->patches_ok || ctx->patches_tried) return XPBD_OK;
    ctx->patches_tried = true;
    if (ctx->wide_palette) return XPBD_OK;  // patch records name a 4-bit palette entry
    const uint32_t C = (uint32_t)ctx->cloths.size();
    std::vector<PatchArrays> per(C);
    std::vector<std::vector<uint32_t>> slot(C);
    std::vector<char> ok(C, 0);
    parallel_for(C, [&](uint32_t k) {
        ClothHost& c = ctx->cloths[k];
        std::vector<uint32_t> si(c.e), sj(c.e), spal(c.e);
        std::vector<float> srest(c.e);
        for (uint32_t q = 0; q < c.e; ++q) {
            si[q] = c.ci[c.perm[q]];
            sj[q] = c.cj[c.perm[q]];
            srest[q] = c.rest[c.perm[q]];
            spal[q] = c.pal_idx[c.perm[q]];
        }
        std::vector<uint32_t> roff, other, eid;
        neighbor_csr(c.n, c.e, si.data(), sj.data(), roff, other, eid);
        ok[k] = build_cloth_patches(c.n, c.rest_pos.data(), c.w.data(), c.e, si.data(), sj.data(), srest.data(),
                                    spal.data(), roff, other, eid, c.vtx_off, k, 256, 4096, per[k], slot[k]);
    });
    for (uint32_t k = 0; k < C; ++k)
        if (!ok[k]) return XPBD_OK;
    PatchArrays patch_arrays;
    std::vector<std::vector<uint32_t>> lambda_patch(C);
    for (uint32_t k = 0; k < C; ++k) {  // append, rebasing offsets into the batch arrays
        const ClothHost& c = ctx->cloths[k];
        PatchArrays& a = patch_arrays;
        const PatchArrays& b = per[k];
        const uint32_t parts0 = (uint32_t)a.parts.size(), con0 = (uint32_t)(a.con.size() / 2),
                       gofs0 = (uint32_t)a.gofs.size(), slots0 = (uint32_t)a.slots.size();
        for (size_t h = 0; h < b.header.size(); h += 6) {
            const uint32_t hd[6] = {b.header[h] + parts0, b.header[h + 1] + con0, b.header[h + 2] + gofs0,
                                    b.header[h + 3], b.header[h + 4], b.header[h + 5]};
            a.header.insert(a.header.end(), hd, hd + 6);
        }
        a.parts.insert(a.parts.end(), b.parts.begin(), b.parts.end());
        a.con.insert(a.con.end(), b.con.begin(), b.con.end());
        for (uint32_t g : b.gofs) a.gofs.push_back(g + slots0);
        a.slots.insert(a.slots.end(), b.slots.begin(), b.slots.end());
        a.max_local = std::max(a.max_local, b.max_local);
        a.max_con = std::max(a.max_con, b.max_con);
        lambda_patch[k].assign(c.e, 0xFFFFFFFFu);
        for (uint32_t q = 0; q < c.e; ++q)
            if (slot[k][q] != 0xFFFFFFFFu) lambda_patch[k][c.perm[q]] = slot[k][q] + con0;
        per[k] = PatchArrays();
    }
    if (patch_arrays.header.empty()) return XPBD_OK;
    const size_t np_ = patch_arrays.header.size() / 6;
    std::vector<XpbdPatch> ph(np_);
    std::vector<uint32_t> words;  // blob storage in u32 words (16-byte = 4 words granularity)
    uint32_t max_blob = 0;
    auto pad16 = [&]() {
        while (words.size() % 4) words.push_back(0);
    };
    for (size_t k = 0; k < np_; ++k) {
        const uint32_t* h = &patch_arrays.header[6 * k];
        const uint32_t parts_off = h[0], con_off = h[1], gofs_off = h[2];
        const uint32_t npo = h[3] & 0xFFFF, nh = h[3] >> 16, nc = h[4];
        const size_t start_w = words.size();
        for (uint32_t t = 0; t < npo + nh; ++t) words.push_back(patch_arrays.parts[parts_off + t]);
        pad16();
        for (uint32_t c = 0; c < nc; ++c) {
            words.push_back(patch_arrays.con[2 * (con_off + c)]);
            words.push_back(patch_arrays.con[2 * (con_off + c) + 1]);
        }
        pad16();
        const uint32_t s0 = patch_arrays.gofs[gofs_off], s1 = patch_arrays.gofs[gofs_off + npo];
        for (uint32_t t = 0; t <= npo; ++t) words.push_back(patch_arrays.gofs[gofs_off + t] - s0);
        pad16();
        for (uint32_t q = s0; q < s1; q += 2) {
            const uint32_t lo = patch_arrays.slots[q];
            const uint32_t hi = (q + 1 < s1) ? patch_arrays.slots[q + 1] : 0u;
            words.push_back(lo | (hi << 16));
        }
        pad16();
        const uint32_t bytes = (uint32_t)((words.size() - start_w) * 4);
        ph[k].off16 = (uint32_t)(start_w / 4);
        ph[k].bytes = bytes;
        ph[k].nc = nc;
        ph[k].lam_off = con_off;
        ph[k].np = (uint16_t)npo;
        ph[k].nh = (uint16_t)nh;
        ph[k].cloth = (uint16_t)h[5];
        ph[k].pad = 0;
        max_blob = std::max(max_blob, bytes);
    }
    const size_t ncon = patch_arrays.con.size() / 2;
    cudaError_t err = cudaSuccess;
    XpbdPatch* d_ph = dev_alloc<XpbdPatch>(ctx, np_, &err);
    if (err != cudaSuccess) return cuda_fail(ctx, err, "cudaMalloc (patches)");
    uint4* d_blob = dev_alloc<uint4>(ctx, words.size() / 4, &err);
    if (err != cudaSuccess) return cuda_fail(ctx, err, "cudaMalloc (patches)");
    float* d_plam = dev_alloc<float>(ctx, ncon, &err);
    if (err != cudaSuccess) return cuda_fail(ctx, err, "cudaMalloc (patches)");
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(d_ph, ph.data(), np_ * sizeof(XpbdPatch), cudaMemcpyHostToDevice, st), "upload");
    CK(cudaMemcpyAsync(d_blob, words.data(), words.size() * 4, cudaMemcpyHostToDevice, st), "upload");
    CK(cudaMemsetAsync(d_plam, 0, std::max<size_t>(ncon, 1) * 4, st), "memset");
    CK(cudaStreamSynchronize(st), "patch upload");
    XpbdWorld& W = ctx->W;
    W.n_patches = (uint32_t)np_;
    W.patch_max_local = patch_arrays.max_local;
    W.patch_max_con = std::max<uint32_t>(patch_arrays.max_con, 1);
    W.patch_con_total = (uint32_t)ncon;
    W.patch_max_blob = max_blob;
    W.patches = d_ph;
    W.patch_blob = d_blob;
    W.patch_lambda = d_plam;
    for (uint32_t k = 0; k < C; ++k) ctx->cloths[k].lambda_patch.swap(lambda_patch[k]);
    ctx->patches_ok = true;
    *usable = true;
    return XPBD_OK;
}

// Gauss–Seidel strips: the packed particles split over `strips` clusters of `cl` CTAs (consecutive ranges); the
// particles joined by a constraint to another strip are kept in global memory slots. Built (or rebuilt for another
// shape) when selected; false if the shape does not fit (the schedule then uses the single-cluster or grid kernel).
static bool build_strip_table(xpbd_ctx* ctx, uint32_t cl, uint32_t strips) {
    if (ctx->strip_cl == cl && ctx->strip_s == strips) return true;
    const uint32_t N = ctx->W.n, ncta = cl * strips, ncol = ctx->W.n_colors;
    if (N == 0 || ncol == 0) return false;
    const uint32_t q = (N + ncta - 1) / ncta;
    if (q > 4096 || q * (ncta - 1) >= N) return false;  // every CTA owns particles
    const uint32_t block = std::min<uint32_t>(512, std::max<uint32_t>(128, (q + 127) / 128 * 128));
    if (!strip_gs_supported(cl, strips, block, q)) {
        cudaGetLastError();
        return false;
    }
    const std::vector<uint4>& con = ctx->con_host;
    auto cta = [q](uint32_t p) { return p / q; };
    auto strip = [q, cl](uint32_t p) { return p / q / cl; };
    std::vector<uint32_t> slot(N, 0xFFFFFFFFu);
    std::vector<uint8_t> bnd(N, 0);
    for (const uint4& r : con)
        if (strip(r.x) != strip(r.y)) slot[r.x] = slot[r.y] = 0u;
    uint32_t ns = 0;
    for (uint32_t p = 0; p < N; ++p)
        if (slot[p] == 0u) slot[p] = ns++;
    const auto shared = [&](uint32_t p) { return slot[p] != 0xFFFFFFFFu; };
    for (const uint4& r : con)
        if (cta(r.x) != cta(r.y)) bnd[r.x] = bnd[r.y] = 1;
    auto kind = [&](const uint4& r) -> uint32_t {
        if (shared(r.x) || shared(r.y)) return 0;
        if (cta(r.x) != cta(r.y) || bnd[r.x] || bnd[r.y]) return 1;
        return 2;
    };
    auto code = [&](uint32_t p) {
        return shared(p) ? (0x80000000u | slot[p]) : (((cta(p) % cl) << 16) | (p - cta(p) * q));
    };
    std::vector<uint32_t> off((size_t)ncol * ncta * 3 + 1, 0);
    for (uint32_t c = 0; c < ncol; ++c)
        for (uint32_t e = ctx->color_off_host[c]; e < ctx->color_off_host[c + 1]; ++e)
            ++off[((size_t)c * ncta + cta(con[e].x)) * 3 + kind(con[e]) + 1];
    for (size_t k = 1; k < off.size(); ++k) off[k] += off[k - 1];
    std::vector<uint32_t> cur(off.begin(), off.end() - 1);
    std::vector<uint4> rec(con.size());
    // CTAs touching each shared particle: its owner and the solvers of its constraints
    std::vector<std::vector<uint32_t>> touch(ns);
    for (uint32_t p = 0; p < N; ++p)
        if (shared(p)) touch[slot[p]].push_back(cta(p));
    for (uint32_t c = 0; c < ncol; ++c)
        for (uint32_t e = ctx->color_off_host[c]; e < ctx->color_off_host[c + 1]; ++e) {
            const uint4 r = con[e];
            rec[cur[((size_t)c * ncta + cta(r.x)) * 3 + kind(r)]++] = make_uint4(code(r.x), code(r.y), r.z, r.w);
            if (shared(r.x)) touch[slot[r.x]].push_back(cta(r.x));
            if (shared(r.y)) touch[slot[r.y]].push_back(cta(r.x));
        }
    std::vector<std::vector<uint32_t>> dep(ncta);
    for (auto& t : touch) {
        std::sort(t.begin(), t.end());
        t.erase(std::unique(t.begin(), t.end()), t.end());
        for (uint32_t a : t)
            for (uint32_t b : t)
                if (a / cl != b / cl) dep[a].push_back(b);
    }
    std::vector<uint32_t> deps, dep_off(ncta + 1, 0);
    for (uint32_t a = 0; a < ncta; ++a) {
        std::sort(dep[a].begin(), dep[a].end());
        dep[a].erase(std::unique(dep[a].begin(), dep[a].end()), dep[a].end());
        deps.insert(deps.end(), dep[a].begin(), dep[a].end());
        dep_off[a + 1] = (uint32_t)deps.size();
    }
    cudaError_t err = cudaSuccess;
    uint4* d_rec = dev_alloc<uint4>(ctx, std::max<size_t>(1, rec.size()), &err);
    uint32_t* d_off = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, off.size(), &err) : nullptr;
    uint32_t* d_slot = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, N, &err) : nullptr;
    float4* d_gx = err == cudaSuccess ? dev_alloc<float4>(ctx, std::max<uint32_t>(1, ns), &err) : nullptr;
    unsigned* d_flags = err == cudaSuccess ? dev_alloc<unsigned>(ctx, ncta, &err) : nullptr;
    uint32_t* d_deps = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, std::max<size_t>(1, deps.size()), &err) : nullptr;
    uint32_t* d_dep_off = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, dep_off.size(), &err) : nullptr;
    if (err != cudaSuccess) return false;
    if (cudaMemcpy(d_rec, rec.data(), rec.size() * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_slot, slot.data(), (size_t)N * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(d_flags, 0, ncta * 4) != cudaSuccess ||
        (!deps.empty() && cudaMemcpy(d_deps, deps.data(), deps.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) ||
        cudaMemcpy(d_dep_off, dep_off.data(), dep_off.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        return false;
    ctx->strip = StripTable{d_rec, d_off, d_slot, d_gx, d_flags, d_deps, d_dep_off, q, ncta, ncol};
    ctx->strip_cl = cl;
    ctx->strip_s = strips;
    ctx->strip_block = block;
    return true;
}

// Strips for Gauss–Seidel (λ cleared per iteration, no collision): `want` strips, or none when 0 / 1.
static bool pick_strips(xpbd_ctx* ctx, uint32_t want) {
    if (ctx->opts.solver != XPBD_SOLVER_GAUSS_SEIDEL || ctx->opts.lambda_mode != XPBD_LAMBDA_RESET_PER_ITERATION ||
        ctx->opts.collision != XPBD_COLLISION_NONE || want < 2)
        return false;
    for (uint32_t cl : {16u, 8u}) {
        if (ctx->opts.cluster_ctas > 1 && ctx->opts.cluster_ctas != cl) continue;
        if (build_strip_table(ctx, cl, want)) return true;
    }
    return false;
}

// Cluster path: Gauss–Seidel, λ cleared per iteration, every particle fits in the cluster's shared memory.
static uint32_t pick_cluster(xpbd_ctx* ctx, uint32_t want, uint32_t block) {
    if (ctx->opts.solver != XPBD_SOLVER_GAUSS_SEIDEL || ctx->opts.lambda_mode != XPBD_LAMBDA_RESET_PER_ITERATION)
        return 0;
    if (want == 1) return 0;
    const uint32_t cands[2] = {16, 8};
    for (uint32_t cl : cands) {
        if (want && want != cl) continue;
        if (ctx->W.n > cl * 16384u) continue;
        if (!build_cluster_table(ctx, cl)) continue;
        if (cluster_gs_supported(cl, ctx->ct.shift, ctx->ct.max_chunk, block)) return cl;
        cudaGetLastError();
    }
    return 0;
}

// Spatial patches for jacobi_kernel 2, built now if needed; false if they cannot be used (the schedule then runs the
// thread-per-particle kernel and the reason is kept in last_error).
static bool patches_usable(xpbd_ctx* ctx) {
    bool usable = false;
    if (ensure_patches(ctx, &usable) != XPBD_OK) return false;
    if (!usable) ctx->last_error = "spatial patches unavailable for this batch: thread-per-particle Jacobi used";
    return usable;
}

// Tables of the cloth-resident Jacobi kernel, built on its first selection. Usable when every cloth fits a cluster
// (8 CTAs of XPBD_CLOTH_RANK_MAX particles, or 16 of 4,096 where the device runs such clusters) and its color
// batches are particle-disjoint (then each
// particle's neighbour-table row is ordered by color, which the kernel's summation order relies on); otherwise the
// schedule keeps the thread-per-particle kernel and the reason is left in last_error.
static int ensure_cloth_tables(xpbd_ctx* ctx, bool* usable) {
    *usable = ctx->cloth_ok;
    if (ctx->cloth_tried) return XPBD_OK;
    ctx->cloth_tried = true;
    const uint32_t C = (uint32_t)ctx->cloths.size();
    std::vector<int> cls(C, -1);
    std::vector<uint32_t> q(C, 0), ncol(C, 0);
    std::vector<std::vector<uint32_t>> seg(C);
    std::vector<std::vector<uint2>> rec(C);
    std::vector<std::vector<float>> comp(C);
    std::atomic<int> bad{0};  // 1: a cloth too large, 2: batches share a particle
    bool class_ok[kClothClasses];
    CK(cloth_kernel_prepare(), "cloth kernel attributes");
    for (int t = 0; t < kClothClasses; ++t) class_ok[t] = cloth_class_launchable(t);
    parallel_for(C, [&](uint32_t k) {
        const ClothHost& c = ctx->cloths[k];
        int id = -1;
        for (int t = 0; t < kClothClasses; ++t)
            if ((uint64_t)kClothClass[t].cl * kClothClass[t].rank_cap >= c.n && class_ok[t]) {
                id = t;
                break;
            }
        if (id < 0) {
            bad = 1;
            return;
        }
        const uint32_t cl = kClothClass[id].cl;
        const uint32_t qq = std::max<uint32_t>(1, (c.n + cl - 1) / cl);
        const uint32_t nb = (uint32_t)c.batch_off.size() - 1;
        std::vector<uint32_t> stamp(c.n, 0xFFFFFFFFu);
        for (uint32_t b = 0; b < nb; ++b)
            for (uint32_t t = c.batch_off[b]; t < c.batch_off[b + 1]; ++t) {
                const uint32_t e = c.perm[t], i = c.ci[e], j = c.cj[e];
                if (stamp[i] == b || (j != i && stamp[j] == b)) {
                    bad = 2;
                    return;
                }
                stamp[i] = b;
                stamp[j] = b;
            }
        // records of constraints with an unpinned endpoint, grouped by (batch, rank owning endpoint i)
        std::vector<uint32_t>& sg = seg[k];
        sg.assign((size_t)nb * cl + 1, 0);
        for (uint32_t b = 0; b < nb; ++b)
            for (uint32_t t = c.batch_off[b]; t < c.batch_off[b + 1]; ++t) {
                const uint32_t e = c.perm[t];
                if (c.w[c.ci[e]] <= 0.f && c.w[c.cj[e]] <= 0.f) continue;
                ++sg[(size_t)b * cl + c.ci[e] / qq + 1];
            }
        for (size_t x = 1; x < sg.size(); ++x) sg[x] += sg[x - 1];
        std::vector<uint32_t> cur(sg.begin(), sg.end() - 1);
        rec[k].resize(sg.back());
        comp[k].resize(sg.back());
        const uint32_t eb = cloth_ep_bits(cl);
        auto ep = [qq, eb](uint32_t p) { return ((p / qq) << eb) | (p % qq); };
        for (uint32_t b = 0; b < nb; ++b)
            for (uint32_t t = c.batch_off[b]; t < c.batch_off[b + 1]; ++t) {
                const uint32_t e = c.perm[t];
                if (c.w[c.ci[e]] <= 0.f && c.w[c.cj[e]] <= 0.f) continue;
                const uint32_t at = cur[(size_t)b * cl + c.ci[e] / qq]++;
                uint32_t rb;
                memcpy(&rb, &c.rest[e], 4);
                rec[k][at] = make_uint2(ep(c.ci[e]) | (ep(c.cj[e]) << 16), rb);
                comp[k][at] = c.comp[e];
            }
        cls[k] = id;
        q[k] = qq;
        ncol[k] = nb;
    });
    if (bad) {
        ctx->last_error = bad == 1 ? "cloth-resident Jacobi: a cloth exceeds a cluster's shared memory"
                                   : "cloth-resident Jacobi: a color batch shares a particle";
        return XPBD_OK;
    }
    // concatenate in cloth order
    std::vector<XpbdClothDesc> desc(C);
    std::vector<size_t> rbase(C + 1, 0), sbase(C + 1, 0);
    for (uint32_t k = 0; k < C; ++k) {
        rbase[k + 1] = rbase[k] + rec[k].size();
        sbase[k + 1] = sbase[k] + seg[k].size();
    }
    if (rbase[C] >= 0xFFFFFFFFull || sbase[C] >= 0xFFFFFFFFull) {
        ctx->last_error = "cloth-resident Jacobi: more than 2^32 records";
        return XPBD_OK;
    }
    std::vector<uint2> all_rec(rbase[C]);
    std::vector<float> all_comp(rbase[C]);
    std::vector<uint32_t> all_seg(sbase[C]);
    parallel_for(C, [&](uint32_t k) {
        const ClothHost& c = ctx->cloths[k];
        std::copy(rec[k].begin(), rec[k].end(), all_rec.begin() + rbase[k]);
        std::copy(comp[k].begin(), comp[k].end(), all_comp.begin() + rbase[k]);
        for (size_t x = 0; x < seg[k].size(); ++x) all_seg[sbase[k] + x] = (uint32_t)(seg[k][x] + rbase[k]);
        desc[k] = XpbdClothDesc{c.vtx_off, c.n, q[k], ncol[k], (uint32_t)sbase[k], kClothClass[cls[k]].cl, {0, 0}};
    });
    // one launch per class, largest cloths first
    std::vector<uint32_t> order;
    uint32_t count[kClothClasses] = {0}, first[kClothClasses] = {0}, cap[kClothClasses] = {0};
    for (int t = 0; t < kClothClasses; ++t) {
        first[t] = (uint32_t)order.size();
        std::vector<uint32_t> mine;
        for (uint32_t k = 0; k < C; ++k)
            if (cls[k] == t) mine.push_back(k);
        std::stable_sort(mine.begin(), mine.end(),
                         [&](uint32_t a, uint32_t b) { return ctx->cloths[a].n > ctx->cloths[b].n; });
        for (uint32_t k : mine) cap[t] = std::max(cap[t], q[k]);
        count[t] = (uint32_t)mine.size();
        order.insert(order.end(), mine.begin(), mine.end());
    }
    cudaError_t err = cudaSuccess;
    XpbdClothDesc* d_desc = dev_alloc<XpbdClothDesc>(ctx, C, &err);
    uint32_t* d_seg = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, all_seg.size(), &err) : nullptr;
    uint2* d_rec = err == cudaSuccess ? dev_alloc<uint2>(ctx, all_rec.size(), &err) : nullptr;
    float* d_comp = err == cudaSuccess ? dev_alloc<float>(ctx, all_comp.size(), &err) : nullptr;
    uint32_t* d_order = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, order.size(), &err) : nullptr;
    if (err != cudaSuccess) return cuda_fail(ctx, err, "cloth-resident tables");
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(d_desc, desc.data(), C * sizeof(XpbdClothDesc), cudaMemcpyHostToDevice, st), "upload");
    CK(cudaMemcpyAsync(d_seg, all_seg.data(), all_seg.size() * 4, cudaMemcpyHostToDevice, st), "upload");
    if (!all_rec.empty()) {
        CK(cudaMemcpyAsync(d_rec, all_rec.data(), all_rec.size() * sizeof(uint2), cudaMemcpyHostToDevice, st),
           "upload");
        CK(cudaMemcpyAsync(d_comp, all_comp.data(), all_comp.size() * 4, cudaMemcpyHostToDevice, st), "upload");
    }
    CK(cudaMemcpyAsync(d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice, st), "upload");
    CK(cudaStreamSynchronize(st), "upload sync");
    CK(cloth_kernel_prepare(), "cloth kernel attributes");
    for (int t = 0; t < kClothClasses; ++t) {
        ctx->cloth_tab[t] = ClothSolveTable{d_desc, d_seg, d_rec, d_comp, d_order + first[t], count[t], cap[t]};
        if (!ctx->cls_stream[t]) CK(cudaStreamCreateWithFlags(&ctx->cls_stream[t], cudaStreamNonBlocking), "stream");
        if (!ctx->ev_join[t]) CK(cudaEventCreateWithFlags(&ctx->ev_join[t], cudaEventDisableTiming), "event");
    }
    if (!ctx->ev_fork) CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "event");
    ctx->cloth_ok = true;
    *usable = true;
    return XPBD_OK;
}

// Tables of the single-cluster small-batch kernel: the rows of the neighbour table split over the cluster's ranks
// (records {self, other endpoint, rest, compliance}), built on its first selection from the device tables.
constexpr uint32_t kSmallBatchMaxParticles = 16 * 512;
static int ensure_small_batch(xpbd_ctx* ctx, bool* usable) {
    const uint32_t want = ctx->opts.cluster_ctas > 1 ? ctx->opts.cluster_ctas : 0u;
    if (ctx->small_tried && (want == 0 || want == ctx->small_cl || !ctx->small_ok)) {
        *usable = ctx->small_ok && (want == 0 || want == ctx->small_cl);
        return XPBD_OK;
    }
    *usable = false;
    ctx->small_tried = true;
    ctx->small_ok = false;
    const uint32_t N = ctx->W.n, C = (uint32_t)ctx->cloths.size();
    if (N == 0 || N > kSmallBatchMaxParticles) return XPBD_OK;
    std::vector<uint32_t> roff(N + 1);
    std::vector<uint2> inc(ctx->W.n_inc);
    std::vector<float> pal((size_t)C * XPBD_PALETTE), icomp(ctx->wide_palette ? ctx->W.n_inc : 0);
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(roff.data(), ctx->W.row_off, (N + 1) * 4, cudaMemcpyDeviceToHost, st), "download");
    if (!inc.empty())
        CK(cudaMemcpyAsync(inc.data(), ctx->W.inc, inc.size() * 8, cudaMemcpyDeviceToHost, st), "download");
    CK(cudaMemcpyAsync(pal.data(), ctx->W.palette_comp, pal.size() * 4, cudaMemcpyDeviceToHost, st), "download");
    if (!icomp.empty())
        CK(cudaMemcpyAsync(icomp.data(), ctx->W.inc_comp, icomp.size() * 4, cudaMemcpyDeviceToHost, st), "download");
    CK(cudaStreamSynchronize(st), "download sync");
    std::vector<uint32_t> cloth_of(N);
    for (uint32_t k = 0; k < C; ++k)
        for (uint32_t i = 0; i < ctx->cloths[k].n; ++i) cloth_of[ctx->cloths[k].vtx_off + i] = k;
    for (uint32_t cl : {16u, 8u}) {
        if (ctx->opts.cluster_ctas > 1 && ctx->opts.cluster_ctas != cl) continue;  // a requested cluster size
        const uint32_t q = (N + cl - 1) / cl;
        if (q > 1024) continue;
        std::vector<uint4> rec;
        std::vector<uint32_t> lroff((size_t)cl * (q + 1), 0), rbase(cl + 1, 0);
        uint32_t m_max = 0, longest = 1;
        // A constraint with both endpoints on one rank is one record (solved once, both endpoint terms written);
        // a constraint between ranks, or towards a pinned particle (whose row is empty), is a record of the free
        // endpoint's row alone. The k-th incidence of row p towards o and the k-th of row o towards p are the same
        // constraint (both rows list their constraints in table order), which pairs up repeated constraints.
        auto slot_in_row = [&](uint32_t row, uint32_t toward, uint32_t nth) {
            for (uint32_t t = roff[row]; t < roff[row + 1]; ++t)
                if ((inc[t].x & XPBD_OTHER_MASK) == toward && nth-- == 0) return t - roff[row];
            return 0xFFFFFFFFu;
        };
        bool paired = true;
        for (uint32_t r = 0; r < cl; ++r) {
            rbase[r] = (uint32_t)rec.size();
            const uint32_t p0 = r * q, p1 = std::min(N, p0 + q);
            for (uint32_t p = p0; p < p1; ++p) {
                lroff[(size_t)r * (q + 1) + (p - p0)] = roff[p] - roff[p0];
                for (uint32_t k = roff[p]; k < roff[p + 1]; ++k) {
                    const uint32_t o = inc[k].x & XPBD_OTHER_MASK;
                    uint32_t slot = 0xFFFFFFFFu;  // the constraint's slot in row o when that row is on this rank
                    if (o >= p0 && o < p1) {
                        uint32_t nth = 0;  // occurrence of o among the earlier incidences of row p
                        for (uint32_t t = roff[p]; t < k; ++t) nth += (inc[t].x & XPBD_OTHER_MASK) == o;
                        slot = slot_in_row(o, p, nth);
                    }
                    if (slot != 0xFFFFFFFFu && o < p) continue;  // recorded from row o
                    const float comp = ctx->wide_palette ? icomp[k]
                                                         : pal[(size_t)cloth_of[p] * XPBD_PALETTE + (inc[k].x >> 28)];
                    uint32_t cb;
                    memcpy(&cb, &comp, 4);
                    uint32_t code = ((o / q) << 12) | (o % q);
                    if (slot != 0xFFFFFFFFu) {
                        if (slot > 0x7FFFu) paired = false;  // (cannot happen: longest <= 0x7FFF is required below)
                        code |= 0x80000000u | ((slot & 0x7FFFu) << 16);
                    }
                    rec.push_back(make_uint4((p - p0) | ((k - roff[p]) << 16), code, inc[k].y, cb));
                }
                longest = std::max(longest, roff[p + 1] - roff[p]);
            }
            const uint32_t m = (uint32_t)rec.size() - rbase[r];
            const uint32_t deg_total = p1 > p0 ? roff[p1] - roff[p0] : 0u;
            for (uint32_t p = (p1 > p0 ? p1 - p0 : 0); p <= q; ++p) lroff[(size_t)r * (q + 1) + p] = deg_total;
            m_max = std::max(m_max, m);
        }
        rbase[cl] = (uint32_t)rec.size();
        const uint32_t block = std::min<uint32_t>(1024, std::max<uint32_t>(32, (std::max(m_max, q) + 31) / 32 * 32));
        const uint32_t stride = (longest + 3u) / 4u * 4u + 1u;  // odd; the kernel reads stride - 1 slots per row
        if (!paired || m_max > 4096 || longest > 0x7FFFu || !small_batch_supported(cl, block, q, m_max, stride)) {
            cudaGetLastError();
            continue;
        }
        cudaError_t err = cudaSuccess;
        uint4* d_rec = dev_alloc<uint4>(ctx, std::max<size_t>(1, rec.size()), &err);
        uint32_t* d_roff = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, lroff.size(), &err) : nullptr;
        uint32_t* d_rbase = err == cudaSuccess ? dev_alloc<uint32_t>(ctx, cl + 1, &err) : nullptr;
        if (err != cudaSuccess) return cuda_fail(ctx, err, "small-batch tables");
        if (!rec.empty())
            CK(cudaMemcpyAsync(d_rec, rec.data(), rec.size() * 16, cudaMemcpyHostToDevice, st), "upload");
        CK(cudaMemcpyAsync(d_roff, lroff.data(), lroff.size() * 4, cudaMemcpyHostToDevice, st), "upload");
        CK(cudaMemcpyAsync(d_rbase, rbase.data(), (cl + 1) * 4, cudaMemcpyHostToDevice, st), "upload");
        CK(cudaStreamSynchronize(st), "upload sync");
        ctx->small = SmallBatch{d_rec, d_roff, d_rbase, q, m_max, stride};
        ctx->small_cl = cl;
        ctx->small_block = block;
        ctx->small_ok = true;
        *usable = true;
        return XPBD_OK;
    }
    return XPBD_OK;
}

static bool small_batch_usable(xpbd_ctx* ctx) {
    bool usable = false;
    if (ensure_small_batch(ctx, &usable) != XPBD_OK) return false;
    return usable;
}

static bool cloth_kernel_usable(xpbd_ctx* ctx) {
    bool usable = false;
    if (ensure_cloth_tables(ctx, &usable) != XPBD_OK) return false;
    return usable;
}

// Launches the frame of the cloth-resident kernel: the class launches fork off the context stream onto their own
// streams (largest class on the context stream itself) and join back.
static cudaError_t launch_cloth_frame(xpbd_ctx* ctx, uint32_t substeps, cudaStream_t st, uint64_t* launches) {
    cudaError_t e = cudaEventRecord(ctx->ev_fork, st);
    if (e != cudaSuccess) return e;
    bool on_main = false;
    for (int t = kClothClasses - 1; t >= 0; --t) {
        const ClothSolveTable& T = ctx->cloth_tab[t];
        if (T.count == 0) continue;
        cudaStream_t s = on_main ? ctx->cls_stream[t] : st;
        if (on_main) {
            e = cudaStreamWaitEvent(s, ctx->ev_fork, 0);
            if (e != cudaSuccess) return e;
        }
        e = launch_cloth_jacobi(t, ctx->W, T, substeps, s);
        *launches += 1;
        if (e != cudaSuccess) return e;
        if (on_main) {
            e = cudaEventRecord(ctx->ev_join[t], s);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ctx->ev_join[t], 0);
            if (e != cudaSuccess) return e;
        }
        on_main = true;
    }
    return cudaSuccess;
}

static void choose_schedule(xpbd_ctx* ctx) {
    uint32_t block = ctx->opts.block_threads ? ctx->opts.block_threads : 256;
    if (block != 128 && block != 256 && block != 512 && block != 1024) block = 256;
    const uint32_t cblock = ctx->opts.block_threads ? block : 1024;
    if (pick_strips(ctx, ctx->opts.gs_strips)) {
        ctx->kernel = 9;
        ctx->cl = 0;
        ctx->block = ctx->strip_block;
        ctx->grid = ctx->strip.ncta;
        ctx->coop = false;
        ctx->stats.grid_blocks = ctx->strip.ncta;
        ctx->stats.block_threads = ctx->strip_block;
        ctx->stats.solver_kernel = 9;
        ctx->stats.cluster_ctas = ctx->strip_cl;
        return;
    }
    ctx->cl = pick_cluster(ctx, ctx->opts.cluster_ctas, cblock);
    if (ctx->cl) {
        ctx->kernel = 1;
        ctx->block = cblock;
        ctx->grid = ctx->cl;
        ctx->coop = false;
        ctx->stats.grid_blocks = ctx->cl;
        ctx->stats.block_threads = cblock;
        ctx->stats.solver_kernel = 3;
        ctx->stats.cluster_ctas = ctx->cl;
        return;
    }
    const bool plain_jacobi = ctx->opts.solver == XPBD_SOLVER_JACOBI && !(ctx->opts.tolerance > 0.f) &&
                              !ctx->opts.warm_start;
    const bool cloth_eligible = plain_jacobi && ctx->opts.lambda_mode == XPBD_LAMBDA_RESET_PER_ITERATION &&
                                ctx->opts.collision == XPBD_COLLISION_NONE;
    const bool small_default = ctx->opts.jacobi_kernel == 0 && ctx->W.n <= 4096;
    if (cloth_eligible && (small_default || ctx->opts.jacobi_kernel == 5) && small_batch_usable(ctx)) {
        ctx->kernel = 8;
        ctx->block = ctx->small_block;
        ctx->grid = ctx->small_cl;
        ctx->coop = false;
        ctx->stats.grid_blocks = ctx->small_cl;
        ctx->stats.block_threads = ctx->small_block;
        ctx->stats.solver_kernel = 8;
        ctx->stats.cluster_ctas = ctx->small_cl;
        return;
    }
    if (cloth_eligible && ctx->opts.jacobi_kernel == 4 && cloth_kernel_usable(ctx)) {
        ctx->kernel = 7;
        uint32_t blocks = 0, maxcl = 1;
        for (int t = 0; t < kClothClasses; ++t) {
            blocks += ctx->cloth_tab[t].count * kClothClass[t].cl;
            if (ctx->cloth_tab[t].count) maxcl = std::max(maxcl, kClothClass[t].cl);
        }
        ctx->block = 1024;
        ctx->grid = blocks;
        ctx->coop = false;
        ctx->stats.grid_blocks = blocks;
        ctx->stats.block_threads = 1024;
        ctx->stats.solver_kernel = 7;
        ctx->stats.cluster_ctas = maxcl;
        return;
    }
    if (ctx->opts.solver == XPBD_SOLVER_JACOBI && (ctx->opts.tolerance > 0.f || ctx->opts.warm_start))
        ctx->kernel = 6;
    else if (ctx->opts.solver == XPBD_SOLVER_GAUSS_SEIDEL)
        ctx->kernel = 1;
    else if (ctx->opts.jacobi_kernel == 1)
        ctx->kernel = 0;
    else if (ctx->opts.jacobi_kernel == 2 && patches_usable(ctx))
        ctx->kernel = 2;
    else
        ctx->kernel = 5;  // thread per particle (default): measured fastest on the sheets and batches benchmarked
    int maxb = max_blocks_per_sm(ctx->kernel, block, ctx->W);
    if (maxb < 1) maxb = 1;
    int bps = ctx->opts.blocks_per_sm ? (int)ctx->opts.blocks_per_sm : maxb;
    if (bps > maxb) bps = maxb;
    // never more blocks than useful work
    uint64_t need;
    if (ctx->kernel == 0) need = ((uint64_t)ctx->W.n_tiles * 32 + block - 1) / block;
    else if (ctx->kernel == 2) need = ctx->W.n_patches;
    else need = ((uint64_t)ctx->W.n + block - 1) / block;  // rows / convergence solve: thread per particle
    uint32_t grid = (uint32_t)ctx->sms * (uint32_t)bps;
    if (grid > need) grid = (uint32_t)std::max<uint64_t>(1, need);
    ctx->block = block;
    ctx->grid = grid;
    ctx->coop = ctx->coop_supported;
    ctx->stats.grid_blocks = grid;
    ctx->stats.block_threads = block;
    ctx->stats.solver_kernel = ctx->kernel;
    ctx->stats.cluster_ctas = 0;
}

static cudaError_t launch_substeps(xpbd_ctx* ctx, uint32_t flags, uint32_t substeps, uint32_t pend, uint32_t start,
                                   cudaStream_t st) {
    if (ctx->cl)
        return launch_cluster_gs(ctx->cl, ctx->block, ctx->W, ctx->ct, flags, substeps, pend, st);
    return launch_solver(ctx->kernel, ctx->block, ctx->grid, ctx->coop, ctx->W, flags, substeps, pend, start, st);
}

static int ensure_collision_buffers(xpbd_ctx* ctx) {
    const xpbd_solver_opts& o = ctx->opts;
    const uint32_t N = ctx->W.n;
    cudaError_t err = cudaSuccess;
    if (!ctx->coll_ready || ctx->cb.table_bits != o.hash_table_bits) {
        if (o.hash_table_bits < 4 || o.hash_table_bits > 28)
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "hash_table_bits must be in [4, 28]");
        CollisionBuffers& B = ctx->cb;
        B.table_bits = o.hash_table_bits;
        B.keys = dev_alloc<uint32_t>(ctx, N, &err);
        if (err == cudaSuccess) B.vals = dev_alloc<uint32_t>(ctx, N, &err);
        if (err == cudaSuccess) B.keys_sorted = dev_alloc<uint32_t>(ctx, N, &err);
        if (err == cudaSuccess) B.vals_sorted = dev_alloc<uint32_t>(ctx, N, &err);
        if (err == cudaSuccess) B.table = dev_alloc<uint2>(ctx, (size_t)1 << B.table_bits, &err);
        if (err == cudaSuccess) B.pos_sorted = dev_alloc<float4>(ctx, N, &err);
        if (err == cudaSuccess) B.pair_count = dev_alloc<uint32_t>(ctx, N + 1, &err);
        B.sort_scratch_bytes = radix_sort_scratch_bytes(N);
        if (err == cudaSuccess) B.sort_scratch = dev_alloc<char>(ctx, B.sort_scratch_bytes, &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "collision buffers");
        // every entry empty, and a valid "previous build" of key 0 for the first build to clear
        CK(cudaMemsetAsync(B.table, 0xFF, ((size_t)1 << B.table_bits) * sizeof(uint2), ctx->stream), "memset");
        CK(cudaMemsetAsync(B.keys_sorted, 0, (size_t)N * 4, ctx->stream), "memset");
        ctx->coll_ready = true;
    }
    if (o.collision == XPBD_COLLISION_RING_FILTER && ctx->coll_ring_depth_built != o.ring_depth) {
        std::vector<uint32_t> off, idx;
        for (auto& c : ctx->cloths)
            topology_rings(c.n, c.e, c.ci.data(), c.cj.data(), c.ctype.data(), o.ring_depth, c.vtx_off, off, idx);
        uint32_t* doff = dev_alloc<uint32_t>(ctx, off.size(), &err);
        uint32_t* didx = nullptr;
        if (err == cudaSuccess) didx = dev_alloc<uint32_t>(ctx, idx.size(), &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "ring buffers");
        CK(cudaMemcpyAsync(doff, off.data(), off.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload");
        if (!idx.empty())
            CK(cudaMemcpyAsync(didx, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, ctx->stream), "upload");
        CK(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->cb.ring_off = doff;
        ctx->cb.ring_idx = didx;
        ctx->coll_ring_depth_built = o.ring_depth;
    }
    return XPBD_OK;
}

// Learned warm start: features → MLP → λ0 per incidence (defined with the MLP host code below).
cudaError_t launch_mlp_warm_start(xpbd_ctx* ctx, cudaStream_t st, uint64_t* launches);

// Enqueues one frame (opts.substeps substeps) on `st`. Returns the number of kernel launches.
static cudaError_t enqueue_frame(xpbd_ctx* ctx, cudaStream_t st, uint64_t* launches) {
    const xpbd_solver_opts& o = ctx->opts;
    const uint32_t S = std::max<uint32_t>(1, o.substeps);
    const uint32_t I = ctx->tsp.inner_iterations;
    const uint32_t solver = o.solver;
    const bool coll = o.collision != XPBD_COLLISION_NONE && o.coll_scale > 1e-12f;
    const uint32_t every = std::max<uint32_t>(1, o.collision_every_n_substeps);
    const float inv_cell = ctx->hp.inv_cell;
    cudaError_t e;
    if (ctx->kernel == 6) {  // convergence solve: per substep predict, [λ0], solve-to-tolerance + finalize
        const uint32_t warm = o.warm_start;
        for (uint32_t s = 0; s < S; ++s) {
            e = launch_converge_predict(ctx->W, ctx->sms, st);
            *launches += 1;
            if (e != cudaSuccess) return e;
            if (warm == XPBD_WARM_PREVIOUS && ctx->W.n_inc) {
                e = cudaMemcpyAsync(ctx->W.warm_lam_inc, ctx->W.inc_lambda, (size_t)ctx->W.n_inc * 4,
                                    cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return e;
            } else if (warm == XPBD_WARM_LEARNED) {
                e = launch_mlp_warm_start(ctx, st, launches);
                if (e != cudaSuccess) return e;
            }
            e = launch_solver(6, ctx->block, ctx->grid, ctx->coop, ctx->W, warm ? 1u : 0u, 1, 0, 0, st);
            *launches += 1;
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    if (ctx->kernel == 7) return launch_cloth_frame(ctx, S, st, launches);  // no collision (choose_schedule)
    if (ctx->kernel == 8) {
        *launches += 1;
        return launch_small_batch(ctx->small_cl, ctx->small_block, ctx->W, ctx->small, S, st);
    }
    if (ctx->kernel == 9) {  // no collision (pick_strips)
        *launches += 1;
        return launch_strip_gs(ctx->strip_cl, ctx->strip_block, ctx->W, ctx->strip, S, st);
    }
    if (!coll) {
        e = launch_substeps(ctx, kEndFinalize, S, 0, 0, st);
        *launches += 1;
        return e;
    }
    bool pending = false;
    uint32_t pend = 0;
    for (uint32_t s = 0; s < S; ++s) {
        const bool run_coll = (s % every) == every - 1;
        const bool last = s + 1 == S;
        uint32_t flags = pending ? kBeginFinalize : 0u;
        if (last && !run_coll) flags |= kEndFinalize;
        const uint32_t start = (solver == XPBD_SOLVER_JACOBI) ? pend : 0u;
        e = launch_substeps(ctx, flags, 1, pend, start, st);
        *launches += 1;
        if (e != cudaSuccess) return e;
        if (last && !run_coll) return cudaSuccess;
        const uint32_t fin = (solver == XPBD_SOLVER_JACOBI) ? ((start + I) & 1u) : 0u;
        if (run_coll) {
            e = collision_build(ctx->W, ctx->W.jac[fin], ctx->cb, inv_cell, ctx->sms, st, launches);
            if (e != cudaSuccess) return e;
            e = collision_resolve(ctx->W, ctx->W.jac[fin], ctx->W.jac[fin ^ 1u], ctx->cb, inv_cell, o.collision,
                                  ctx->sms, st, launches);
            if (e != cudaSuccess) return e;
            pend = fin ^ 1u;
        } else {
            pend = fin;
        }
        pending = true;
    }
    e = launch_finalize(ctx->W, pend, ctx->sms, st);
    *launches += 1;
    return e;
}

static std::string schedule_key(xpbd_ctx* ctx) {
    const xpbd_solver_opts& o = ctx->opts;
    char buf[256];
    snprintf(buf, sizeof(buf), "%u/%u/%u/%u/%u/%u/%u/%u/%d/%p/%u/%u/%u/%u/%u/%u/%u", o.solver, o.substeps,
             o.collision, o.collision_every_n_substeps, ctx->tsp.inner_iterations, ctx->block, ctx->grid,
             (int)ctx->coop, (int)(o.coll_scale > 1e-12f), (void*)ctx->stream, o.hash_table_bits, o.ring_depth,
             ctx->cl, ctx->kernel, o.warm_start, ctx->strip_cl, ctx->strip_s);
    return buf;
}

bool mlp_ready(xpbd_ctx* ctx);

static int check_ready(xpbd_ctx* ctx) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "xpbd_commit has not been called");
    if (!ctx->params_set) return fail(ctx, XPBD_ERR_STATE, "xpbd_set_params has not been called");
    return XPBD_OK;
}

extern "C" int xpbd_set_params(xpbd_ctx* ctx, const xpbd_time_step_params* params, const xpbd_solver_opts* opts) {
    if (!ctx || !params) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "xpbd_commit has not been called");
    if (!(params->dt > 0.f) || !std::isfinite(params->inv_dt))
        return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "dt must be positive");
    if (opts) {
        if (opts->solver > XPBD_SOLVER_GAUSS_SEIDEL || opts->relaxation > XPBD_RELAX_AVERAGE ||
            opts->lambda_mode > XPBD_LAMBDA_PER_SUBSTEP || opts->collision > XPBD_COLLISION_RING_FILTER)
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "unknown solver option value");
        if (opts->collision != XPBD_COLLISION_NONE && !(opts->hash_cell >= opts->thickness))
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "hash_cell must be >= thickness");
        if (opts->warm_start > XPBD_WARM_PREVIOUS) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad warm_start");
        const bool converge = opts->tolerance > 0.f || opts->warm_start;
        if (converge && opts->solver != XPBD_SOLVER_JACOBI)
            return fail(ctx, XPBD_ERR_UNSUPPORTED, "the convergence solve is a Jacobi solve");
        if (converge && opts->collision != XPBD_COLLISION_NONE)
            return fail(ctx, XPBD_ERR_UNSUPPORTED, "the convergence solve has no collision pass");
        if (converge && params->inner_iterations > XPBD_MAX_CONVERGE_ITERS)
            return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "convergence solve: at most 4096 iterations per substep");
        if (opts->warm_start == XPBD_WARM_LEARNED && !mlp_ready(ctx))
            return fail(ctx, XPBD_ERR_STATE, "learned warm start needs a trained or loaded MLP (xpbd_mlp_*)");
        ctx->opts = *opts;
    }
    ctx->tsp = *params;
    fill_dev_params(ctx);
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(ctx->dparams, &ctx->hp, sizeof(XpbdDevParams), cudaMemcpyHostToDevice, ctx->stream),
       "params upload");
    if (ctx->opts.collision != XPBD_COLLISION_NONE) {
        int r = ensure_collision_buffers(ctx);
        if (r != XPBD_OK) return r;
    }
    choose_schedule(ctx);
    ctx->params_set = true;
    return XPBD_OK;
}

// Errors with which the runtime refuses a cooperative launch (as opposed to a failure of the work itself).
static bool coop_refused(cudaError_t e) {
    return e == cudaErrorCooperativeLaunchTooLarge || e == cudaErrorNotSupported ||
           e == cudaErrorStreamCaptureUnsupported || e == cudaErrorNotPermitted;
}

static int run_frames(xpbd_ctx* ctx, uint32_t frames) {
    cudaStream_t st = ctx->stream;
    if (ctx->opts.use_graphs) {
        std::string key = schedule_key(ctx);
        if (!ctx->exec || key != ctx->graph_key) {
            if (ctx->exec) cudaGraphExecDestroy(ctx->exec);
            ctx->exec = nullptr;
            cudaGraph_t g = nullptr;
            uint64_t launches = 0;
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
            cudaError_t e = enqueue_frame(ctx, st, &launches);
            cudaError_t e2 = cudaStreamEndCapture(st, &g);
            if (e != cudaSuccess || e2 != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                // nothing of a failed capture ran: if the cooperative attribute was refused, capture again without
                // it (the bounded barriers still hold; stats.cooperative_launch then reads 0)
                if (ctx->coop && coop_refused(e != cudaSuccess ? e : e2)) {
                    ctx->coop = false;
                    return run_frames(ctx, frames);
                }
                return cuda_fail(ctx, e != cudaSuccess ? e : e2, "frame graph capture");
            }
            e = cudaGraphInstantiate(&ctx->exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "graph instantiate");
            ctx->graph_key = key;
            ctx->graph_nodes = launches;
        }
        for (uint32_t f = 0; f < frames; ++f) CK(cudaGraphLaunch(ctx->exec, st), "graph launch");
        ctx->stats.kernel_launches += ctx->graph_nodes * frames;
        ctx->stats.graph_captured = 1;
    } else {
        for (uint32_t f = 0; f < frames; ++f) {
            uint64_t launches = 0;
            cudaError_t e = enqueue_frame(ctx, st, &launches);
            // Retry without the cooperative attribute only when the refused launch was the frame's first (the
            // solver launch of every schedule but the convergence solve, which predicts first): then nothing of
            // the frame has been queued and running it again cannot advance the state twice.
            if (e != cudaSuccess && ctx->coop && coop_refused(e) && launches <= 1 && ctx->kernel != 6) {
                cudaGetLastError();
                ctx->coop = false;
                launches = 0;
                e = enqueue_frame(ctx, st, &launches);
            }
            if (e != cudaSuccess) return cuda_fail(ctx, e, "frame launch");
            ctx->stats.kernel_launches += launches;
        }
        ctx->stats.graph_captured = 0;
    }
    ctx->stats.cooperative_launch = ctx->coop ? 1 : 0;
    ctx->stats.frames += frames;
    ctx->stats.substeps += (uint64_t)frames * std::max<uint32_t>(1, ctx->opts.substeps);
    return XPBD_OK;
}

extern "C" int xpbd_step(xpbd_ctx* ctx, uint32_t frames) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return run_frames(ctx, frames);
}

extern "C" int xpbd_step_params(xpbd_ctx* ctx, const xpbd_time_step_params* params, uint32_t frames) {
    int r = xpbd_set_params(ctx, params, nullptr);
    if (r != XPBD_OK) return r;
    return xpbd_step(ctx, frames);
}

extern "C" int xpbd_substep(xpbd_ctx* ctx, uint32_t substeps) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    xpbd_solver_opts saved = ctx->opts;
    ctx->opts.substeps = 1;
    ctx->opts.use_graphs = 0;
    choose_schedule(ctx);
    for (uint32_t s = 0; s < substeps && r == XPBD_OK; ++s) r = run_frames(ctx, 1);
    ctx->stats.frames -= substeps;
    ctx->opts = saved;
    choose_schedule(ctx);
    return r;
}

static int read_status(xpbd_ctx* ctx) {
    int h[4] = {0, 0, 0, 0};
    CK(cudaMemcpyAsync(h, ctx->W.status, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "status read");
    CK(cudaStreamSynchronize(ctx->stream), "stream sync");
    if (h[0] == 0) return XPBD_OK;
    // clear the status and the barrier state so the context stays usable
    CK(cudaMemsetAsync(ctx->W.status, 0, 4 * sizeof(int), ctx->stream), "memset");
    CK(cudaMemsetAsync(ctx->W.sync, 0, sizeof(XpbdGridSync), ctx->stream), "memset");
    if (ctx->strip.flags)  // a strip launch that gave up leaves its step flags uneven: start them over
        CK(cudaMemsetAsync(ctx->strip.flags, 0, ctx->strip.ncta * sizeof(unsigned), ctx->stream), "memset");
    CK(cudaStreamSynchronize(ctx->stream), "stream sync");
    if (h[0] & XPBD_DEV_BARRIER_TIMEOUT) return fail(ctx, XPBD_ERR_BARRIER_TIMEOUT, "grid barrier wait timed out");
    if (h[0] & XPBD_DEV_NONFINITE) return fail(ctx, XPBD_ERR_DEVICE_NONFINITE, "non-finite position or velocity");
    if (h[0] & XPBD_DEV_CAPACITY) return fail(ctx, XPBD_ERR_CAPACITY, "device capacity exceeded");
    return fail(ctx, XPBD_ERR_INDEX_RANGE, "device index out of range");
}

extern "C" int xpbd_sync(xpbd_ctx* ctx) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return XPBD_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return read_status(ctx);
}

// ------------------------------------------------------------------------------------------------- state
__global__ static void pack_xyz_kernel(const float4* __restrict__ src, uint32_t n, float* __restrict__ dst) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p = src[i];
        dst[3 * i] = p.x;
        dst[3 * i + 1] = p.y;
        dst[3 * i + 2] = p.z;
    }
}

static int read_vec(xpbd_ctx* ctx, const float4* src, uint32_t cloth_id, float* out) {
    if (!ctx || !out) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    uint32_t off = 0, n = ctx->W.n;
    if (cloth_id != 0xFFFFFFFFu) {
        if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
        off = ctx->cloths[cloth_id].vtx_off;
        n = ctx->cloths[cloth_id].n;
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    uint32_t grid = std::min<uint32_t>((n + 255) / 256, (uint32_t)ctx->sms * 8);
    pack_xyz_kernel<<<std::max<uint32_t>(grid, 1), 256, 0, ctx->stream>>>(src + off, n, ctx->d_xyz);
    CK(cudaGetLastError(), "pack");
    const size_t bytes = 3 * (size_t)n * sizeof(float);
    if (ctx->pinned && ctx->pinned_bytes >= bytes) {
        CK(cudaMemcpyAsync(ctx->pinned, ctx->d_xyz, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
        int r = read_status(ctx);
        memcpy(out, ctx->pinned, bytes);
        return r;
    }
    CK(cudaMemcpyAsync(out, ctx->d_xyz, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    return read_status(ctx);
}

extern "C" int xpbd_read_positions(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz) {
    return read_vec(ctx, ctx ? ctx->W.x : nullptr, cloth_id, out_xyz);
}
extern "C" int xpbd_read_velocities(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz) {
    return read_vec(ctx, ctx ? ctx->W.v : nullptr, cloth_id, out_xyz);
}

static int upload_state(xpbd_ctx* ctx, uint32_t cloth_id, const float* xyz, const float* vel, bool from_initial) {
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    for (uint32_t c = 0; c < ctx->cloths.size(); ++c) {
        if (cloth_id != 0xFFFFFFFFu && c != cloth_id) continue;
        ClothHost& h = ctx->cloths[c];
        std::vector<float4> x(h.n), v(h.n);
        for (uint32_t i = 0; i < h.n; ++i) {
            const float* p = from_initial ? &h.pos[3 * i] : (xyz ? &xyz[3 * i] : nullptr);
            const float* q = from_initial ? nullptr : (vel ? &vel[3 * i] : nullptr);
            x[i] = p ? make_float4(p[0], p[1], p[2], h.w[i]) : make_float4(0, 0, 0, h.w[i]);
            v[i] = q ? make_float4(q[0], q[1], q[2], 0.f) : make_float4(0, 0, 0, 0);
        }
        if (from_initial || xyz) {
            if (!from_initial && !xyz) continue;
            CK(cudaMemcpy(ctx->W.x + h.vtx_off, x.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice), "upload");
            CK(cudaMemcpy(ctx->W.jac[0] + h.vtx_off, x.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice), "upload");
            CK(cudaMemcpy(ctx->W.jac[1] + h.vtx_off, x.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice), "upload");
        }
        if (from_initial || vel)
            CK(cudaMemcpy(ctx->W.v + h.vtx_off, v.data(), h.n * sizeof(float4), cudaMemcpyHostToDevice), "upload");
    }
    return XPBD_OK;
}

extern "C" int xpbd_write_state(xpbd_ctx* ctx, uint32_t cloth_id, const float* xyz, const float* vel_xyz) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id != 0xFFFFFFFFu && cloth_id >= ctx->cloths.size())
        return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    if (cloth_id == 0xFFFFFFFFu && ctx->cloths.size() > 1 && (xyz || vel_xyz)) {
        // packed arrays for all cloths
        uint32_t off = 0;
        for (uint32_t c = 0; c < ctx->cloths.size(); ++c) {
            int r = upload_state(ctx, c, xyz ? xyz + 3 * (size_t)off : nullptr,
                                 vel_xyz ? vel_xyz + 3 * (size_t)off : nullptr, false);
            if (r != XPBD_OK) return r;
            off += ctx->cloths[c].n;
        }
        return XPBD_OK;
    }
    return upload_state(ctx, cloth_id, xyz, vel_xyz, false);
}

extern "C" int xpbd_reset(xpbd_ctx* ctx) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    int r = upload_state(ctx, 0xFFFFFFFFu, nullptr, nullptr, true);
    if (r != XPBD_OK) return r;
    CK(cudaMemset(ctx->W.inc_lambda, 0, std::max<size_t>(ctx->W.n_inc, 1) * 4), "memset");
    CK(cudaMemset(ctx->W.con_lambda, 0, std::max<size_t>(ctx->W.e, 1) * 4), "memset");
    if (ctx->W.patch_lambda)
        CK(cudaMemset(ctx->W.patch_lambda, 0, std::max<size_t>(ctx->W.patch_con_total, 1) * 4), "memset");
    return XPBD_OK;
}

extern "C" int xpbd_set_cloth_grab(xpbd_ctx* ctx, uint32_t cloth_id, int32_t vertex, const float* target,
                                   float stiffness) {
    if (!ctx || (vertex >= 0 && !target)) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    const ClothHost& c = ctx->cloths[cloth_id];
    if (vertex >= (int32_t)c.n) return fail(ctx, XPBD_ERR_INDEX_RANGE, "grab vertex out of range");
    XpbdGrab g{-1, {0.f, 0.f, 0.f}, 0.f, {0u, 0u, 0u}};
    if (vertex >= 0) {
        g.idx = (int32_t)(c.vtx_off + (uint32_t)vertex);
        g.target[0] = target[0];
        g.target[1] = target[1];
        g.target[2] = target[2];
        g.stiffness = stiffness;
    }
    ctx->grabs[cloth_id] = g;
    uint32_t active = 0;
    for (const XpbdGrab& h : ctx->grabs) active += h.idx >= 0 ? 1u : 0u;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    // ordered with the frames on the context's stream; the host copies are staged before the calls return
    CK(cudaMemcpyAsync(const_cast<XpbdGrab*>(ctx->W.grabs) + cloth_id, &ctx->grabs[cloth_id], sizeof(XpbdGrab), cudaMemcpyHostToDevice,
                       ctx->stream), "grab");
    CK(cudaMemcpyAsync(const_cast<uint32_t*>(ctx->W.grab_count), &active, sizeof(uint32_t), cudaMemcpyHostToDevice,
                       ctx->stream), "grab");
    CK(cudaStreamSynchronize(ctx->stream), "grab");
    return XPBD_OK;
}

extern "C" int xpbd_set_cloth_wind(xpbd_ctx* ctx, uint32_t cloth_id, const float* velocity, float drag) {
    if (!ctx || (drag != 0.f && !velocity)) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    if (!(drag >= 0.f) || !std::isfinite(drag)) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "wind drag must be >= 0");
    XpbdWind w{{0.f, 0.f, 0.f}, 0.f};
    if (drag > 0.f) {
        w.vel[0] = velocity[0];
        w.vel[1] = velocity[1];
        w.vel[2] = velocity[2];
        w.drag = drag;
    }
    ctx->winds[cloth_id] = w;
    uint32_t active = 0;
    for (const XpbdWind& h : ctx->winds) active += h.drag > 0.f ? 1u : 0u;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    // ordered with the frames on the context's stream; the host copies are staged before the call returns
    CK(cudaMemcpyAsync(const_cast<XpbdWind*>(ctx->W.winds) + cloth_id, &ctx->winds[cloth_id], sizeof(XpbdWind),
                       cudaMemcpyHostToDevice, ctx->stream), "wind");
    CK(cudaMemcpyAsync(const_cast<uint32_t*>(ctx->W.wind_count), &active, sizeof(uint32_t), cudaMemcpyHostToDevice,
                       ctx->stream), "wind");
    CK(cudaStreamSynchronize(ctx->stream), "wind");
    return XPBD_OK;
}

extern "C" int xpbd_read_normals(xpbd_ctx* ctx, uint32_t cloth_id, float* out_xyz) {
    if (!ctx || !out_xyz) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    if (ctx->W.n_tris == 0) return fail(ctx, XPBD_ERR_STATE, "no triangles: xpbd_set_triangles before xpbd_commit");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(launch_vertex_normals(ctx->W, ctx->sms, ctx->stream), "normals");
    ctx->stats.kernel_launches += 1;
    return read_vec(ctx, ctx->W.normals, cloth_id, out_xyz);
}

extern "C" int xpbd_read_lambda(xpbd_ctx* ctx, uint32_t cloth_id, float* out) {
    if (!ctx || !out) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const ClothHost& h = ctx->cloths[cloth_id];
    const uint32_t kern = (ctx->kernel >= 5) ? 0u : ctx->kernel;  // rows / convergence solve: incidence λ
    const float* src = kern == 0 ? ctx->W.inc_lambda : (kern == 2 ? ctx->W.patch_lambda : ctx->W.con_lambda);
    const size_t cnt = kern == 0 ? ctx->W.n_inc : (kern == 2 ? ctx->W.patch_con_total : ctx->W.e);
    std::vector<float> all(std::max<size_t>(cnt, 1));
    if (cnt) CK(cudaMemcpyAsync(all.data(), src, cnt * 4, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    int r = read_status(ctx);
    const std::vector<uint32_t>& map = kern == 0 ? h.lambda_inc : (kern == 2 ? h.lambda_patch : h.lambda_gs);
    for (uint32_t e = 0; e < h.e; ++e) out[e] = map[e] == 0xFFFFFFFFu ? 0.f : all[map[e]];
    return r;
}

extern "C" int xpbd_strain_residual(xpbd_ctx* ctx, uint32_t cloth_id, float* out) {
    if (!ctx || !out) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    uint32_t e0 = 0, e1 = ctx->W.e;
    if (cloth_id != 0xFFFFFFFFu) {
        if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
        e0 = ctx->cloths[cloth_id].con_off;
        e1 = e0 + ctx->cloths[cloth_id].e;
    }
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaMemsetAsync(ctx->d_resid, 0, 4, ctx->stream), "memset");
    if (e1 > e0) CK(launch_strain_residual(ctx->W, e0, e1, ctx->d_resid, ctx->sms, ctx->stream), "residual");
    unsigned bits = 0;
    CK(cudaMemcpyAsync(&bits, ctx->d_resid, 4, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    int r = read_status(ctx);
    memcpy(out, &bits, 4);
    return r;
}

extern "C" int xpbd_get_stats(xpbd_ctx* ctx, xpbd_stats* out) {
    if (!ctx || !out) return XPBD_ERR_INVALID_ARGUMENT;
    if (ctx->committed) {
        XpbdConvergeStats cs{};
        CK(cudaSetDevice(ctx->device), "cudaSetDevice");
        CK(cudaMemcpyAsync(&cs, ctx->W.cstats, sizeof(cs), cudaMemcpyDeviceToHost, ctx->stream), "stats");
        CK(cudaStreamSynchronize(ctx->stream), "stats");
        ctx->stats.converge_iterations = cs.iterations;
        ctx->stats.converge_substeps = cs.substeps;
        ctx->stats.converge_max_iterations = cs.max_iterations;
        ctx->stats.warm_start_fallbacks = cs.fallbacks;
    }
    *out = ctx->stats;
    return XPBD_OK;
}

extern "C" int xpbd_converge_history(xpbd_ctx* ctx, float* residuals, uint32_t max_count, uint32_t* count) {
    if (!ctx || !count || (max_count && !residuals)) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    XpbdConvergeStats cs{};
    CK(cudaMemcpyAsync(&cs, ctx->W.cstats, sizeof(cs), cudaMemcpyDeviceToHost, ctx->stream), "stats");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    *count = cs.last_iterations;
    const uint32_t n = std::min(max_count, cs.last_iterations);
    if (n) {
        CK(cudaMemcpyAsync(residuals, ctx->W.iter_res, n * 4, cudaMemcpyDeviceToHost, ctx->stream), "history");
        CK(cudaStreamSynchronize(ctx->stream), "sync");
    }
    return XPBD_OK;
}

extern "C" int xpbd_converge_cloth_iterations(xpbd_ctx* ctx, uint32_t* out) {
    if (!ctx || !out) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint32_t nc = (uint32_t)ctx->cloths.size();
    if (nc) CK(cudaMemcpyAsync(out, ctx->W.cloth_iters, nc * 4, cudaMemcpyDeviceToHost, ctx->stream), "iters");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return XPBD_OK;
}

extern "C" int xpbd_set_warm_lambda(xpbd_ctx* ctx, uint32_t cloth_id, const float* lambda0) {
    if (!ctx || !lambda0) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const ClothHost& h = ctx->cloths[cloth_id];
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    std::vector<float> all(std::max<uint32_t>(ctx->W.n_inc, 1));
    CK(cudaMemcpy(all.data(), ctx->W.warm_lam_inc, all.size() * 4, cudaMemcpyDeviceToHost), "readback");
    for (uint32_t e = 0; e < h.e; ++e) {
        if (h.inc_i[e] != 0xFFFFFFFFu) all[h.inc_i[e]] = lambda0[e];
        if (h.inc_j[e] != 0xFFFFFFFFu) all[h.inc_j[e]] = lambda0[e];
    }
    CK(cudaMemcpy(ctx->W.warm_lam_inc, all.data(), all.size() * 4, cudaMemcpyHostToDevice), "upload");
    return XPBD_OK;
}

extern "C" int xpbd_get_coloring(xpbd_ctx* ctx, uint32_t cloth_id, uint32_t* perm, uint32_t* offsets,
                                 uint32_t* batch_count) {
    if (!ctx || !batch_count) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    const ClothHost& h = ctx->cloths[cloth_id];
    *batch_count = (uint32_t)h.batch_off.size() - 1;
    if (perm) std::copy(h.perm.begin(), h.perm.end(), perm);
    if (offsets) std::copy(h.batch_off.begin(), h.batch_off.end(), offsets);
    return XPBD_OK;
}

extern "C" int xpbd_color_constraints(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj,
                                      uint32_t order, uint32_t* perm, uint32_t* offsets, uint32_t* batch_count) {
    if (!batch_count || (e_count && (!ci || !cj || !perm || !offsets))) return XPBD_ERR_INVALID_ARGUMENT;
    if (order != XPBD_ORDER_COLOR_REFERENCE && order != XPBD_ORDER_COLOR_INDEX) return XPBD_ERR_INVALID_ARGUMENT;
    for (uint32_t e = 0; e < e_count; ++e)
        if (ci[e] >= n || cj[e] >= n || ci[e] == cj[e]) return XPBD_ERR_INDEX_RANGE;
    std::vector<uint32_t> p, colors, offs;
    color_constraints(n, e_count, ci, cj, order == XPBD_ORDER_COLOR_INDEX, p, colors, offs);
    *batch_count = (uint32_t)offs.size() - 1;
    if (perm) std::copy(p.begin(), p.end(), perm);
    if (offsets) std::copy(offs.begin(), offs.end(), offsets);
    return XPBD_OK;
}

// ------------------------------------------------------------------------------------------------- autotune
extern "C" int xpbd_autotune(xpbd_ctx* ctx, uint32_t frames, xpbd_solver_opts* opts_out) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    // plain Jacobi: the spatial-patch kernel is one of the candidates, so its tables are built now if they are not yet
    // (a batch that cannot be split into patches simply has no patch candidates)
    if (ctx->opts.solver == XPBD_SOLVER_JACOBI && !(ctx->opts.tolerance > 0.f || ctx->opts.warm_start)) {
        bool usable = false;
        r = ensure_patches(ctx, &usable);
        if (r != XPBD_OK) return r;
    }
    const uint32_t N = ctx->W.n;
    float4 *sx = nullptr, *sv = nullptr;
    CK(cudaMalloc(&sx, (size_t)N * sizeof(float4)), "snapshot");
    CK(cudaMalloc(&sv, (size_t)N * sizeof(float4)), "snapshot");
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(sx, ctx->W.x, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "snapshot");
    CK(cudaMemcpyAsync(sv, ctx->W.v, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "snapshot");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    xpbd_solver_opts base = ctx->opts;
    float best = 1e30f;
    xpbd_solver_opts best_opts = base;
    struct Cand {
        uint32_t block, bps, cl, jk, strips;
    };
    std::vector<Cand> cands;
    const uint32_t blocks[] = {128, 256, 512, 1024};
    const uint32_t jks[3] = {2, 3, 1};
    for (uint32_t jk : jks) {
        if (base.solver != XPBD_SOLVER_JACOBI && jk != 1) continue;
        if (jk == 2 && !ctx->patches_ok) continue;
        const uint32_t kid = base.solver == XPBD_SOLVER_JACOBI ? (jk == 2 ? 2u : (jk == 3 ? 5u : 0u)) : 1u;
        for (uint32_t blk : blocks) {
            int maxb = max_blocks_per_sm(kid, blk, ctx->W);
            for (int bps = 1; bps <= maxb; bps *= 2) cands.push_back({blk, (uint32_t)bps, 1, jk, 1});
        }
    }
    if (base.solver == XPBD_SOLVER_JACOBI && !(base.tolerance > 0.f || base.warm_start) &&
        base.lambda_mode == XPBD_LAMBDA_RESET_PER_ITERATION && base.collision == XPBD_COLLISION_NONE &&
        cloth_kernel_usable(ctx))
        cands.push_back({0, 0, 1, 4, 1});  // cloth-resident kernel (its launch shapes are fixed per cloth size)
    if (base.solver == XPBD_SOLVER_JACOBI && !(base.tolerance > 0.f || base.warm_start) &&
        base.lambda_mode == XPBD_LAMBDA_RESET_PER_ITERATION && base.collision == XPBD_COLLISION_NONE &&
        small_batch_usable(ctx))
        cands.push_back({0, 0, 1, 5, 1});  // the whole batch in one cluster
    if (base.solver == XPBD_SOLVER_GAUSS_SEIDEL && base.cluster_ctas != 1) {
        for (uint32_t cl : {16u, 8u})
            for (uint32_t blk : {512u, 1024u}) cands.push_back({blk, 0, cl, 0, 1});
        if (base.gs_strips != 1 && base.lambda_mode == XPBD_LAMBDA_RESET_PER_ITERATION &&
            base.collision == XPBD_COLLISION_NONE && ctx->W.n >= 16384)
            for (uint32_t strips : {2u, 4u, 8u}) cands.push_back({0, 0, 16, 0, strips});
    }
    for (const Cand& cd : cands) {
        ctx->opts = base;
        ctx->opts.block_threads = cd.block;
        ctx->opts.blocks_per_sm = cd.bps;
        ctx->opts.cluster_ctas = cd.cl;
        ctx->opts.jacobi_kernel = cd.jk;
        ctx->opts.gs_strips = cd.strips;
        choose_schedule(ctx);
        if (cd.strips > 1 && ctx->kernel != 9) continue;             // strip shape not launchable here
        if (cd.strips <= 1 && cd.cl > 1 && ctx->cl != cd.cl) continue;  // cluster candidate not launchable here
        r = run_frames(ctx, 1);  // warm-up / capture
        if (r != XPBD_OK) break;
        cudaEventRecord(a, st);
        r = run_frames(ctx, std::max<uint32_t>(1, frames));
        cudaEventRecord(b, st);
        if (r != XPBD_OK) break;
        r = read_status(ctx);
        if (r != XPBD_OK) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) {
            best = ms;
            best_opts = ctx->opts;
        }
        CK(cudaMemcpyAsync(ctx->W.x, sx, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "restore");
        CK(cudaMemcpyAsync(ctx->W.v, sv, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "restore");
    }
    CK(cudaMemcpyAsync(ctx->W.x, sx, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "restore");
    CK(cudaMemcpyAsync(ctx->W.v, sv, (size_t)N * 16, cudaMemcpyDeviceToDevice, st), "restore");
    cudaStreamSynchronize(st);
    cudaFree(sx);
    cudaFree(sv);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->opts = (r == XPBD_OK) ? best_opts : base;
    choose_schedule(ctx);
    if (opts_out) *opts_out = ctx->opts;
    return r;
}

// ------------------------------------------------------------------------------------------------- collision
extern "C" int xpbd_collision_keys(xpbd_ctx* ctx, uint32_t* keys, uint32_t* sorted_keys, uint32_t* sorted_vals) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    r = ensure_collision_buffers(ctx);
    if (r != XPBD_OK) return r;
    uint64_t launches = 0;
    CK(collision_build(ctx->W, ctx->W.x, ctx->cb, ctx->hp.inv_cell, ctx->sms, ctx->stream, &launches), "build");
    const size_t bytes = (size_t)ctx->W.n * 4;
    if (keys) CK(cudaMemcpyAsync(keys, ctx->cb.keys, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    if (sorted_keys)
        CK(cudaMemcpyAsync(sorted_keys, ctx->cb.keys_sorted, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    if (sorted_vals)
        CK(cudaMemcpyAsync(sorted_vals, ctx->cb.vals_sorted, bytes, cudaMemcpyDeviceToHost, ctx->stream), "readback");
    return read_status(ctx);
}

extern "C" int xpbd_collision_pairs(xpbd_ctx* ctx, uint32_t* pairs, uint64_t cap, uint64_t* count) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    if (!count) return XPBD_ERR_INVALID_ARGUMENT;
    if (ctx->opts.collision == XPBD_COLLISION_NONE) return fail(ctx, XPBD_ERR_STATE, "collision is off");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    r = ensure_collision_buffers(ctx);
    if (r != XPBD_OK) return r;
    uint64_t launches = 0;
    CK(collision_build(ctx->W, ctx->W.x, ctx->cb, ctx->hp.inv_cell, ctx->sms, ctx->stream, &launches), "build");
    uint32_t* dpairs = nullptr;
    uint64_t cap_d = 0;
    uint64_t total = 0;
    // first pass counts; then allocate and write
    CK(collision_pairs(ctx->W, ctx->W.x, ctx->cb, ctx->hp.inv_cell, ctx->opts.collision, nullptr, 0, &total,
                       ctx->sms, ctx->stream), "pair count");
    *count = total;
    ctx->stats.collision_pairs = total;
    if (pairs && cap > 0 && total > 0) {
        cap_d = std::min<uint64_t>(cap, total);
        CK(cudaMalloc(&dpairs, cap_d * 8), "pairs");
        uint64_t t2 = 0;
        cudaError_t e = collision_pairs(ctx->W, ctx->W.x, ctx->cb, ctx->hp.inv_cell, ctx->opts.collision, dpairs,
                                        cap_d, &t2, ctx->sms, ctx->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(pairs, dpairs, cap_d * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        cudaFree(dpairs);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pair write");
    }
    return read_status(ctx);
}

// ------------------------------------------------------------------------------------------------- primitives
bool xpbd_sort_arrays_overlap(const void* keys_in, const void* vals_in, const void* keys_out, const void* vals_out,
                              uint32_t n);
extern "C" size_t xpbd_radix_sort_scratch_bytes(uint32_t n) { return radix_sort_scratch_bytes(n); }

extern "C" int xpbd_radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, uint32_t n, uint32_t passes, void* scratch,
                                     size_t scratch_bytes, void* stream) {
    if (n && (!keys_in || !vals_in || !keys_out || !vals_out || !scratch)) return XPBD_ERR_INVALID_ARGUMENT;
    if (passes < 1 || passes > 4) return XPBD_ERR_INVALID_ARGUMENT;
    if (n > XPBD_RADIX_SORT_MAX_KEYS) return XPBD_ERR_CAPACITY;
    if (scratch_bytes < radix_sort_scratch_bytes(n)) return XPBD_ERR_INVALID_ARGUMENT;
    if (n && xpbd_sort_arrays_overlap(keys_in, vals_in, keys_out, vals_out, n)) return XPBD_ERR_INVALID_ARGUMENT;
    cudaError_t e = radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, n, passes, scratch, scratch_bytes,
                                     (cudaStream_t)stream, nullptr);
    return e == cudaSuccess ? XPBD_OK : XPBD_ERR_CUDA;
}

extern "C" int xpbd_hash_keys(const float* xyzw, uint32_t n, float inv_cell, uint32_t table_bits, uint32_t* keys,
                              void* stream) {
    if (n && (!xyzw || !keys)) return XPBD_ERR_INVALID_ARGUMENT;
    if (table_bits < 1 || table_bits > 32) return XPBD_ERR_INVALID_ARGUMENT;
    cudaError_t e = launch_hash_keys((const float4*)xyzw, n, inv_cell, table_bits, keys, nullptr,
                                     (cudaStream_t)stream);
    return e == cudaSuccess ? XPBD_OK : XPBD_ERR_CUDA;
}

// ------------------------------------------------------------------------------------------------- warm-start MLP
bool mlp_ready(xpbd_ctx* ctx) { return ctx && ctx->d_mlp != nullptr; }

cudaError_t launch_mlp_warm_start(xpbd_ctx* ctx, cudaStream_t st, uint64_t* launches) {
    *launches += 1;
    return launch_mlp_infer(ctx->W, ctx->d_mlp, ctx->sms, st);
}

static int mlp_upload_norm(xpbd_ctx* ctx) {
    XpbdMlp* m = ctx->d_mlp;
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    CK(cudaMemcpy(m->fmean, ctx->norm, 9 * 4, cudaMemcpyHostToDevice), "norm");
    CK(cudaMemcpy(m->fstd, ctx->norm + 9, 9 * 4, cudaMemcpyHostToDevice), "norm");
    CK(cudaMemcpy(&m->tmean, ctx->norm + 18, 4, cudaMemcpyHostToDevice), "norm");
    CK(cudaMemcpy(&m->tstd, ctx->norm + 19, 4, cudaMemcpyHostToDevice), "norm");
    return XPBD_OK;
}

extern "C" int xpbd_mlp_init(xpbd_ctx* ctx, uint64_t seed, uint32_t capacity) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->committed) return fail(ctx, XPBD_ERR_STATE, "not committed");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaError_t err = cudaSuccess;
    if (!ctx->d_mlp) {
        ctx->d_mlp = dev_alloc<XpbdMlp>(ctx, 1, &err);
        if (err == cudaSuccess) ctx->d_master = dev_alloc<float>(ctx, XPBD_MLP_PARAMS, &err);
        if (err == cudaSuccess) ctx->d_m1 = dev_alloc<float>(ctx, XPBD_MLP_PARAMS, &err);
        if (err == cudaSuccess) ctx->d_m2 = dev_alloc<float>(ctx, XPBD_MLP_PARAMS, &err);
        if (err == cudaSuccess) ctx->d_grads = dev_alloc<float>(ctx, XPBD_MLP_PARAMS, &err);
        if (err == cudaSuccess) ctx->d_loss = dev_alloc<float>(ctx, 4096, &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "mlp buffers");
    }
    if (capacity > ctx->ds_cap) {
        CK(cudaStreamSynchronize(ctx->stream), "sync");  // no launch may still use the old buffers
        dev_release(ctx, ctx->d_feat);
        dev_release(ctx, ctx->d_scale);
        dev_release(ctx, ctx->d_target);
        ctx->d_feat = ctx->d_scale = ctx->d_target = nullptr;
        ctx->ds_cap = 0;
        ctx->d_feat = dev_alloc<float>(ctx, (size_t)capacity * 9, &err);
        if (err == cudaSuccess) ctx->d_scale = dev_alloc<float>(ctx, capacity, &err);
        if (err == cudaSuccess) ctx->d_target = dev_alloc<float>(ctx, capacity, &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "mlp dataset");
        ctx->ds_cap = capacity;
    }
    ctx->ds_count = 0;
    ctx->adam_step = 0;
    // seeded uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases (splitmix64 stream)
    std::vector<float> p(XPBD_MLP_PARAMS, 0.f);
    uint64_t z = seed ? seed : 0x9E3779B97F4A7C15ull;
    auto rnd = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        uint64_t x = z;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        x ^= x >> 31;
        return (float)((double)(x >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    for (int k = 0; k < 576; ++k) p[k] = rnd() / sqrtf(9.f);
    for (int k = 0; k < 4096; ++k) p[640 + k] = rnd() / sqrtf(64.f);
    for (int k = 0; k < 64; ++k) p[640 + 4096 + 64 + k] = rnd() / sqrtf(64.f);
    CK(cudaMemcpy(ctx->d_master, p.data(), XPBD_MLP_PARAMS * 4, cudaMemcpyHostToDevice), "mlp init");
    CK(cudaMemset(ctx->d_m1, 0, XPBD_MLP_PARAMS * 4), "mlp init");
    CK(cudaMemset(ctx->d_m2, 0, XPBD_MLP_PARAMS * 4), "mlp init");
    for (int k = 0; k < 9; ++k) {
        ctx->norm[k] = 0.f;
        ctx->norm[9 + k] = 1.f;
    }
    ctx->norm[18] = 0.f;
    ctx->norm[19] = 1.f;
    int r = mlp_upload_norm(ctx);
    if (r != XPBD_OK) return r;
    CK(launch_mlp_publish(ctx->d_master, ctx->d_mlp, ctx->stream), "mlp publish");
    CK(cudaStreamSynchronize(ctx->stream), "mlp init");
    return XPBD_OK;
}

extern "C" int xpbd_mlp_set_params(xpbd_ctx* ctx, const float* params, const float* norm) {
    if (!ctx || !params) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    CK(cudaMemcpy(ctx->d_master, params, XPBD_MLP_PARAMS * 4, cudaMemcpyHostToDevice), "mlp params");
    if (norm) {
        memcpy(ctx->norm, norm, sizeof(ctx->norm));
        int r = mlp_upload_norm(ctx);
        if (r != XPBD_OK) return r;
    }
    CK(launch_mlp_publish(ctx->d_master, ctx->d_mlp, ctx->stream), "mlp publish");
    CK(cudaStreamSynchronize(ctx->stream), "mlp params");
    return XPBD_OK;
}

extern "C" int xpbd_mlp_get_params(xpbd_ctx* ctx, float* params, float* norm) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    if (params) CK(cudaMemcpy(params, ctx->d_master, XPBD_MLP_PARAMS * 4, cudaMemcpyDeviceToHost), "mlp params");
    if (norm) memcpy(norm, ctx->norm, sizeof(ctx->norm));
    return XPBD_OK;
}

extern "C" int xpbd_mlp_predict_lambda(xpbd_ctx* ctx, uint32_t cloth_id, float* out) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    if (!out) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    if (cloth_id >= ctx->cloths.size()) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "bad cloth id");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(launch_converge_predict(ctx->W, ctx->sms, ctx->stream), "predict");
    CK(launch_mlp_infer(ctx->W, ctx->d_mlp, ctx->sms, ctx->stream), "infer");
    ctx->stats.kernel_launches += 2;
    std::vector<float> all(std::max<uint32_t>(ctx->W.n_inc, 1));
    if (ctx->W.n_inc)
        CK(cudaMemcpyAsync(all.data(), ctx->W.warm_lam_inc, ctx->W.n_inc * 4, cudaMemcpyDeviceToHost, ctx->stream),
           "readback");
    r = read_status(ctx);
    const ClothHost& h = ctx->cloths[cloth_id];
    for (uint32_t e = 0; e < h.e; ++e)
        out[e] = h.inc_i[e] != 0xFFFFFFFFu ? all[h.inc_i[e]] : (h.inc_j[e] != 0xFFFFFFFFu ? all[h.inc_j[e]] : 0.f);
    return r;
}

extern "C" int xpbd_mlp_collect(xpbd_ctx* ctx, uint32_t substeps, uint32_t stride) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    if (stride == 0) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "stride must be >= 1");
    if (ctx->kernel != 6) return fail(ctx, XPBD_ERR_STATE, "collection runs the convergence solve: set tolerance > 0");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    const uint32_t warm = ctx->opts.warm_start;
    cudaError_t e = cudaSuccess;
    for (uint32_t s = 0; s < substeps && e == cudaSuccess; ++s) {
        const uint32_t offset = ctx->collect_offset++ % stride;
        const uint32_t avail = ctx->W.e > offset ? (ctx->W.e - offset + stride - 1) / stride : 0;
        const uint32_t take = std::min(avail, ctx->ds_cap - ctx->ds_count);
        uint64_t launches = 0;
        e = launch_converge_predict(ctx->W, ctx->sms, st);
        ++launches;
        // features see the predicted positions and the previous substep's λ, before any warm start
        if (e == cudaSuccess && take) {
            e = launch_mlp_collect_features(ctx->W, stride, offset, ctx->d_feat, ctx->d_scale, ctx->ds_count,
                                            ctx->ds_count + take, st);
            ++launches;
        }
        if (e == cudaSuccess && warm == XPBD_WARM_PREVIOUS && ctx->W.n_inc)
            e = cudaMemcpyAsync(ctx->W.warm_lam_inc, ctx->W.inc_lambda, (size_t)ctx->W.n_inc * 4,
                                cudaMemcpyDeviceToDevice, st);
        else if (e == cudaSuccess && warm == XPBD_WARM_LEARNED)
            e = launch_mlp_warm_start(ctx, st, &launches);
        if (e == cudaSuccess) {
            e = launch_solver(6, ctx->block, ctx->grid, ctx->coop, ctx->W, warm ? 1u : 0u, 1, 0, 0, st);
            ++launches;
        }
        if (e == cudaSuccess && take) {
            e = launch_mlp_collect_targets(ctx->W, stride, offset, ctx->d_scale, ctx->d_target, ctx->ds_count,
                                           ctx->ds_count + take, st);
            ++launches;
        }
        ctx->ds_count += take;
        ctx->stats.kernel_launches += launches;
        ctx->stats.substeps += 1;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "collect");
    return read_status(ctx);
}

extern "C" int xpbd_mlp_dataset_size(xpbd_ctx* ctx, uint32_t* count) {
    if (!ctx || !count) return XPBD_ERR_INVALID_ARGUMENT;
    *count = ctx->ds_count;
    return XPBD_OK;
}

extern "C" int xpbd_mlp_dataset_read(xpbd_ctx* ctx, uint32_t max_rows, float* features, float* targets,
                                     uint32_t* rows) {
    if (!ctx || !rows) return XPBD_ERR_INVALID_ARGUMENT;
    const uint32_t n = std::min(max_rows, ctx->ds_count);
    *rows = n;
    if (!n) return XPBD_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    if (features) CK(cudaMemcpy(features, ctx->d_feat, (size_t)n * 9 * 4, cudaMemcpyDeviceToHost), "read");
    if (targets) CK(cudaMemcpy(targets, ctx->d_target, (size_t)n * 4, cudaMemcpyDeviceToHost), "read");
    return XPBD_OK;
}

extern "C" int xpbd_mlp_fit_normalization(xpbd_ctx* ctx) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp || ctx->ds_count == 0) return fail(ctx, XPBD_ERR_STATE, "no stored samples");
    const uint32_t n = std::min<uint32_t>(ctx->ds_count, 1u << 20);
    std::vector<float> f((size_t)n * 9), t(n);
    uint32_t rows = 0;
    int r = xpbd_mlp_dataset_read(ctx, n, f.data(), t.data(), &rows);
    if (r != XPBD_OK) return r;
    for (int k = 0; k < 5; ++k) {
        double s = 0, s2 = 0;
        for (uint32_t i = 0; i < n; ++i) {
            s += f[(size_t)i * 9 + k];
            s2 += (double)f[(size_t)i * 9 + k] * f[(size_t)i * 9 + k];
        }
        const double mean = s / n, var = std::max(s2 / n - mean * mean, 0.0);
        ctx->norm[k] = (float)mean;
        ctx->norm[9 + k] = (float)std::max(std::sqrt(var), 1e-12);
    }
    for (int k = 5; k < 9; ++k) {
        ctx->norm[k] = 0.f;
        ctx->norm[9 + k] = 1.f;
    }
    double s = 0, s2 = 0;  // of the learned quantity, the change t - f1
    for (uint32_t i = 0; i < n; ++i) {
        const double d = (double)t[i] - f[(size_t)i * 9 + 1];
        s += d;
        s2 += d * d;
    }
    const double mean = s / n, var = std::max(s2 / n - mean * mean, 0.0);
    ctx->norm[18] = (float)mean;
    ctx->norm[19] = (float)std::max(std::sqrt(var), 1e-12);
    return mlp_upload_norm(ctx);
}

// Minibatch indices drawn from the stored samples: xorshift64 seeded with `seed`, index = z % count.
static void draw_indices(uint64_t seed, size_t count, uint32_t n, std::vector<uint32_t>& idx) {
    idx.resize(count);
    uint64_t z = seed ^ 0xD1B54A32D192ED03ull;
    for (size_t k = 0; k < count; ++k) {
        z ^= z << 13;
        z ^= z >> 7;
        z ^= z << 17;
        idx[k] = (uint32_t)(z % n);
    }
}

extern "C" int xpbd_mlp_train(xpbd_ctx* ctx, uint32_t steps, uint32_t batch, float lr, uint64_t seed, float* losses) {
    if (!ctx) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp || ctx->ds_count == 0) return fail(ctx, XPBD_ERR_STATE, "no stored samples");
    if (batch == 0 || steps == 0 || steps > 4096) return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "steps in [1, 4096]");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t need = (size_t)steps * batch;
    if (need > ctx->idx_cap) {
        cudaError_t err = cudaSuccess;
        CK(cudaStreamSynchronize(ctx->stream), "sync");
        dev_release(ctx, ctx->d_idx);
        ctx->d_idx = nullptr;
        ctx->idx_cap = 0;
        ctx->d_idx = dev_alloc<uint32_t>(ctx, need, &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "batch indices");
        ctx->idx_cap = (uint32_t)need;
    }
    std::vector<uint32_t> idx;
    draw_indices(seed, need, ctx->ds_count, idx);
    cudaStream_t st = ctx->stream;
    CK(cudaMemcpyAsync(ctx->d_idx, idx.data(), need * 4, cudaMemcpyHostToDevice, st), "indices");
    CK(cudaMemsetAsync(ctx->d_loss, 0, steps * 4, st), "memset");
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (uint32_t s = 0; s < steps; ++s) {
        ++ctx->adam_step;
        CK(cudaMemsetAsync(ctx->d_grads, 0, XPBD_MLP_PARAMS * 4, st), "memset");
        CK(launch_mlp_train(ctx->d_mlp, ctx->d_feat, ctx->d_target, ctx->d_idx + (size_t)s * batch, batch,
                            ctx->d_grads, ctx->d_loss + s, ctx->W.status, st), "train");
        const float bc1 = 1.f - powf(b1, (float)ctx->adam_step), bc2 = 1.f - powf(b2, (float)ctx->adam_step);
        CK(launch_mlp_adam(ctx->d_master, ctx->d_m1, ctx->d_m2, ctx->d_grads, 1.0f, lr, b1, b2, eps, bc1, bc2, ctx->d_mlp,
                           st), "adam");
        ctx->stats.kernel_launches += 3;
    }
    if (losses) {
        CK(cudaMemcpyAsync(losses, ctx->d_loss, steps * 4, cudaMemcpyDeviceToHost, st), "losses");
        CK(cudaStreamSynchronize(st), "sync");
        for (uint32_t s = 0; s < steps; ++s) losses[s] /= (float)batch;
    }
    return read_status(ctx);
}

extern "C" int xpbd_mlp_minibatch_gradients(xpbd_ctx* ctx, uint32_t batch, uint64_t seed, float* grads,
                                            float* loss) {
    if (!ctx || !grads || !loss || batch == 0) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp || ctx->ds_count == 0) return fail(ctx, XPBD_ERR_STATE, "no stored samples");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (batch > ctx->idx_cap) {
        cudaError_t err = cudaSuccess;
        CK(cudaStreamSynchronize(ctx->stream), "sync");
        dev_release(ctx, ctx->d_idx);
        ctx->d_idx = nullptr;
        ctx->idx_cap = 0;
        ctx->d_idx = dev_alloc<uint32_t>(ctx, batch, &err);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "batch indices");
        ctx->idx_cap = batch;
    }
    std::vector<uint32_t> idx;
    draw_indices(seed, batch, ctx->ds_count, idx);
    cudaStream_t st = ctx->stream;
    // the copy must not overwrite indices an earlier launch on this stream still reads
    CK(cudaStreamSynchronize(st), "sync");
    CK(cudaMemcpyAsync(ctx->d_idx, idx.data(), (size_t)batch * 4, cudaMemcpyHostToDevice, st), "indices");
    CK(cudaMemsetAsync(grads, 0, XPBD_MLP_PARAMS * 4, st), "memset");
    CK(cudaMemsetAsync(loss, 0, 4, st), "memset");
    CK(launch_mlp_train(ctx->d_mlp, ctx->d_feat, ctx->d_target, ctx->d_idx, batch, grads, loss, ctx->W.status, st),
       "train");
    ctx->stats.kernel_launches += 1;
    return XPBD_OK;
}

extern "C" int xpbd_mlp_apply_gradients(xpbd_ctx* ctx, const float* grads, float scale, float lr) {
    if (!ctx || !grads) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    ++ctx->adam_step;
    const float bc1 = 1.f - powf(b1, (float)ctx->adam_step), bc2 = 1.f - powf(b2, (float)ctx->adam_step);
    CK(launch_mlp_adam(ctx->d_master, ctx->d_m1, ctx->d_m2, grads, scale, lr, b1, b2, eps, bc1, bc2, ctx->d_mlp,
                       ctx->stream), "adam");
    ctx->stats.kernel_launches += 2;
    return XPBD_OK;
}

extern "C" int xpbd_mlp_eval(xpbd_ctx* ctx, const float* features, uint32_t n, float* out) {
    if (!ctx || (n && (!features || !out))) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    if (!n) return XPBD_OK;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    float *df = nullptr, *dout = nullptr;
    CK(cudaMalloc(&df, (size_t)n * 9 * 4), "eval");
    cudaError_t e = cudaMalloc(&dout, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMemcpyAsync(df, features, (size_t)n * 9 * 4, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_mlp_eval(ctx->d_mlp, df, n, dout, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(df);
    if (dout) cudaFree(dout);
    return e == cudaSuccess ? XPBD_OK : cuda_fail(ctx, e, "eval");
}

extern "C" int xpbd_mlp_gradients(xpbd_ctx* ctx, const float* features, const float* targets, uint32_t n,
                                  float* grads, float* loss) {
    if (!ctx || !n || !features || !targets || !grads) return XPBD_ERR_INVALID_ARGUMENT;
    if (!ctx->d_mlp) return fail(ctx, XPBD_ERR_STATE, "xpbd_mlp_init first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    float *df = nullptr, *dt = nullptr, *dg = nullptr, *dl = nullptr;
    uint32_t* di = nullptr;
    std::vector<uint32_t> idx(n);
    for (uint32_t k = 0; k < n; ++k) idx[k] = k;
    cudaError_t e = cudaMalloc(&df, (size_t)n * 9 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dt, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&di, (size_t)n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dg, XPBD_MLP_PARAMS * 4);
    if (e == cudaSuccess) e = cudaMalloc(&dl, 4);
    cudaStream_t st = ctx->stream;
    if (e == cudaSuccess) e = cudaMemcpyAsync(df, features, (size_t)n * 36, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, targets, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(di, idx.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dg, 0, XPBD_MLP_PARAMS * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dl, 0, 4, st);
    if (e == cudaSuccess) e = launch_mlp_train(ctx->d_mlp, df, dt, di, n, dg, dl, ctx->W.status, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(grads, dg, XPBD_MLP_PARAMS * 4, cudaMemcpyDeviceToHost, st);
    float lsum = 0.f;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&lsum, dl, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    for (void* p : {(void*)df, (void*)dt, (void*)di, (void*)dg, (void*)dl})
        if (p) cudaFree(p);
    if (loss) *loss = lsum / (float)n;
    return e == cudaSuccess ? XPBD_OK : cuda_fail(ctx, e, "gradients");
}

// ------------------------------------------------------------------------------------------------- diagnostics
extern "C" int xpbd_selftest_division(int device, uint64_t count, uint64_t seed, uint64_t* mismatches) {
    if (!mismatches) return XPBD_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device) != cudaSuccess) return XPBD_ERR_NO_DEVICE;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return XPBD_ERR_CUDA;
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess) return XPBD_ERR_OUT_OF_MEMORY;
    cudaError_t e = cudaMemset(d, 0, sizeof(*d));
    if (e == cudaSuccess) e = launch_division_selftest(count, seed, d, sms, 0);
    unsigned long long h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    *mismatches = h;
    return e == cudaSuccess ? XPBD_OK : XPBD_ERR_CUDA;
}

extern "C" const char* xpbd_last_error(xpbd_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

extern "C" const char* xpbd_status_string(int s) {
    switch (s) {
        case XPBD_OK: return "ok";
        case XPBD_ERR_INVALID_ARGUMENT: return "invalid argument";
        case XPBD_ERR_CUDA: return "CUDA error";
        case XPBD_ERR_OUT_OF_MEMORY: return "out of device memory";
        case XPBD_ERR_UNSUPPORTED: return "unsupported";
        case XPBD_ERR_STATE: return "invalid state";
        case XPBD_ERR_DEVICE_NONFINITE: return "non-finite state on device";
        case XPBD_ERR_BARRIER_TIMEOUT: return "grid barrier timeout";
        case XPBD_ERR_INDEX_RANGE: return "index out of range";
        case XPBD_ERR_CAPACITY: return "capacity exceeded";
        case XPBD_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

extern "C" int xpbd_debug_force_barrier_timeout(xpbd_ctx* ctx, float timeout_ms) {
    int r = check_ready(ctx);
    if (r != XPBD_OK) return r;
    if (!(timeout_ms > 0.f) || timeout_ms > 10000.f)
        return fail(ctx, XPBD_ERR_INVALID_ARGUMENT, "timeout must be in (0, 10000] ms");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (ctx->kernel == 7 || ctx->kernel == 8)
        return fail(ctx, XPBD_ERR_UNSUPPORTED, "this schedule has no wait across thread-block clusters to force");
    if (ctx->kernel == 9) {
        // strips: one CTA that waits for others starts from a step count its dependencies never reach
        std::vector<uint32_t> dep_off(ctx->strip.ncta + 1);
        CK(cudaMemcpy(dep_off.data(), ctx->strip.dep_off, dep_off.size() * 4, cudaMemcpyDeviceToHost), "download");
        uint32_t victim = 0xFFFFFFFFu;
        for (uint32_t c = 0; c < ctx->strip.ncta && victim == 0xFFFFFFFFu; ++c)
            if (dep_off[c + 1] > dep_off[c]) victim = c;
        if (victim == 0xFFFFFFFFu) return fail(ctx, XPBD_ERR_UNSUPPORTED, "no strip shares particles");
        const unsigned far = 0x40000000u;
        CK(cudaMemcpyAsync(ctx->strip.flags + victim, &far, 4, cudaMemcpyHostToDevice, ctx->stream), "flags");
        ctx->forced_timeout_ms = timeout_ms;
        fill_dev_params(ctx);
        CK(cudaMemcpyAsync(ctx->dparams, &ctx->hp, sizeof(XpbdDevParams), cudaMemcpyHostToDevice, ctx->stream), "p");
        cudaError_t e = launch_strip_gs(ctx->strip_cl, ctx->strip_block, ctx->W, ctx->strip, 1, ctx->stream);
        ctx->forced_timeout_ms = 0.f;
        fill_dev_params(ctx);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "forced launch");
        r = read_status(ctx);  // expected XPBD_ERR_BARRIER_TIMEOUT; also starts the step flags over
        CK(cudaMemcpyAsync(ctx->dparams, &ctx->hp, sizeof(XpbdDevParams), cudaMemcpyHostToDevice, ctx->stream), "p");
        CK(cudaStreamSynchronize(ctx->stream), "sync");
        return r;
    }
    // one extra expected block: the barrier can never complete and must time out
    XpbdGridSync gs = {0u, 0u, 1u, 0u};
    ctx->forced_timeout_ms = timeout_ms;
    fill_dev_params(ctx);
    CK(cudaMemcpyAsync(ctx->dparams, &ctx->hp, sizeof(XpbdDevParams), cudaMemcpyHostToDevice, ctx->stream), "p");
    CK(cudaMemcpyAsync(ctx->W.sync, &gs, sizeof(gs), cudaMemcpyHostToDevice, ctx->stream), "sync");
    xpbd_solver_opts saved = ctx->opts;
    ctx->opts.use_graphs = 0;
    cudaError_t e = launch_solver(ctx->cl ? 1u : ctx->kernel, ctx->cl ? 256u : ctx->block,
                                  ctx->cl ? (uint32_t)ctx->sms : ctx->grid, ctx->coop_supported, ctx->W, kEndFinalize,
                                  1, 0, 0, ctx->stream);
    ctx->opts = saved;
    ctx->forced_timeout_ms = 0.f;
    fill_dev_params(ctx);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "forced launch");
    (void)saved;
    r = read_status(ctx);  // expected XPBD_ERR_BARRIER_TIMEOUT; also resets the barrier state
    CK(cudaMemcpyAsync(ctx->dparams, &ctx->hp, sizeof(XpbdDevParams), cudaMemcpyHostToDevice, ctx->stream), "p");
    CK(cudaStreamSynchronize(ctx->stream), "sync");
    return r;
}
