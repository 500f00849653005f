// ORACLE C API — test infrastructure only (see xpbd_oracle.hpp). Built into oracle/liboracle.so by
// oracle/build_oracle.py with -O2 -ffp-contract=off; loaded by oracle/oracle.py through ctypes.
#include <cstdio>
#include <memory>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "xpbd_oracle.hpp"

using namespace oracle;

extern "C" {

// ---------------------------------------------------------------------------------------------- mesh prep
struct OracleMesh {
    Mesh m;
};

void* oracle_mesh_grid_hanging(uint32_t quad_cols, uint32_t quad_rows, float cell) {
    auto* h = new OracleMesh;
    h->m = grid_cloth_hanging(quad_cols, quad_rows, cell);
    return h;
}
void* oracle_mesh_parse_obj(const char* text) {
    auto* h = new OracleMesh;
    h->m = parse_welded_obj(std::string(text));
    return h;
}
void oracle_mesh_free(void* h) { delete (OracleMesh*)h; }

// sizes: [num_particles, num_constraints, num_indices, batch_count, num_neighbor_entries]
void oracle_mesh_sizes(void* h, uint32_t* out5) {
    const Mesh& m = ((OracleMesh*)h)->m;
    out5[0] = m.num_particles;
    out5[1] = (uint32_t)m.constraint_i.size();
    out5[2] = (uint32_t)m.indices.size();
    out5[3] = m.constraint_batch_count;
    out5[4] = (uint32_t)m.neighbor_other.size();
}
// Any pointer may be NULL.
void oracle_mesh_get(void* h, float* positions, float* rest_positions, float* inv_mass, uint32_t* indices,
                     uint32_t* ci, uint32_t* cj, float* rest, float* comp, uint32_t* batch_offsets,
                     uint32_t* nb_offsets, uint32_t* nb_other, uint32_t* nb_eid, float* nb_rest, float* nb_comp) {
    const Mesh& m = ((OracleMesh*)h)->m;
    for (size_t i = 0; i < m.positions.size(); ++i) {
        if (positions) {
            positions[3 * i] = m.positions[i].x;
            positions[3 * i + 1] = m.positions[i].y;
            positions[3 * i + 2] = m.positions[i].z;
        }
        if (rest_positions) {
            rest_positions[3 * i] = m.rest_positions[i].x;
            rest_positions[3 * i + 1] = m.rest_positions[i].y;
            rest_positions[3 * i + 2] = m.rest_positions[i].z;
        }
        if (inv_mass) inv_mass[i] = m.inv_mass[i];
    }
    if (indices) std::copy(m.indices.begin(), m.indices.end(), indices);
    if (ci) std::copy(m.constraint_i.begin(), m.constraint_i.end(), ci);
    if (cj) std::copy(m.constraint_j.begin(), m.constraint_j.end(), cj);
    if (rest) std::copy(m.constraint_rest_len.begin(), m.constraint_rest_len.end(), rest);
    if (comp) std::copy(m.constraint_compliance.begin(), m.constraint_compliance.end(), comp);
    if (batch_offsets) std::copy(m.constraint_batch_offsets.begin(), m.constraint_batch_offsets.end(), batch_offsets);
    if (nb_offsets) std::copy(m.neighbor_offsets.begin(), m.neighbor_offsets.end(), nb_offsets);
    if (nb_other) std::copy(m.neighbor_other.begin(), m.neighbor_other.end(), nb_other);
    if (nb_eid) std::copy(m.neighbor_constraint_id.begin(), m.neighbor_constraint_id.end(), nb_eid);
    if (nb_rest) std::copy(m.neighbor_rest_len.begin(), m.neighbor_rest_len.end(), nb_rest);
    if (nb_comp) std::copy(m.neighbor_compliance.begin(), m.neighbor_compliance.end(), nb_comp);
}

// partition_constraints_for_gs_batches on raw constraints. perm_out/colors_out: E entries; offsets_out: E+1
// entries capacity. Returns the batch count.
uint32_t oracle_partition(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, int order_by_index,
                          uint32_t* perm_out, uint32_t* colors_out, uint32_t* offsets_out) {
    std::vector<Constraint> cons(e_count);
    for (uint32_t e = 0; e < e_count; ++e) cons[e] = {ci[e], cj[e], 0.0f, 0.0f};
    Partition p = partition_constraints_for_gs_batches(n, cons, order_by_index != 0);
    std::copy(p.perm.begin(), p.perm.end(), perm_out);
    std::copy(p.colors.begin(), p.colors.end(), colors_out);
    std::copy(p.offsets.begin(), p.offsets.end(), offsets_out);
    return (uint32_t)(p.offsets.size() - 1);
}

void oracle_build_csr(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, uint32_t* off,
                      uint32_t* other, uint32_t* eid) {
    std::vector<uint32_t> a(ci, ci + e_count), b(cj, cj + e_count);
    Csr c = build_neighbor_csr(n, a, b);
    std::copy(c.offsets.begin(), c.offsets.end(), off);
    std::copy(c.other.begin(), c.other.end(), other);
    std::copy(c.eid.begin(), c.eid.end(), eid);
}

// ---------------------------------------------------------------------------------------------- solver
}  // extern "C"

struct OracleSim {
    int fp64;
    Sim<float> f;
    Sim<double> d;
};

template <typename T>
static void sim_init(Sim<T>& s, uint32_t n, const float* x, const float* v, const float* w, const float* rest_pos,
                     uint32_t e_count, const uint32_t* ci, const uint32_t* cj, const float* rest, const float* comp,
                     const uint32_t* ctype) {
    s.n = n;
    s.sim_pos.resize(n);
    s.prev_pos.resize(n);
    s.vel.resize(n);
    s.jac_a.resize(n);
    s.jac_b.resize(n);
    s.rest_pos.resize(n);
    s.inv_mass.resize(n);
    for (uint32_t i = 0; i < n; ++i) {
        s.sim_pos[i] = Sim<T>::cvt(x, i);
        s.prev_pos[i] = {0, 0, 0};
        s.vel[i] = v ? Sim<T>::cvt(v, i) : V3<T>{0, 0, 0};
        s.rest_pos[i] = rest_pos ? Sim<T>::cvt(rest_pos, i) : s.sim_pos[i];
        s.inv_mass[i] = (T)w[i];
    }
    s.ci.assign(ci, ci + e_count);
    s.cj.assign(cj, cj + e_count);
    s.ctype.assign(e_count, 0);
    if (ctype) s.ctype.assign(ctype, ctype + e_count);
    s.rest.resize(e_count);
    s.comp.resize(e_count);
    for (uint32_t e = 0; e < e_count; ++e) {
        s.rest[e] = (T)rest[e];
        s.comp[e] = (T)comp[e];
    }
    s.lambda.assign(e_count, 0);
    s.delta_lambda.assign(e_count, 0);
    Csr c = build_neighbor_csr(n, s.ci, s.cj);
    s.nb_off = c.offsets;
    s.nb_other = c.other;
    s.nb_eid = c.eid;
    // 2-ring over stretch/shear constraints (type 0/1): vertices within two hops, excluding self, sorted.
    std::vector<std::vector<uint32_t>> adj(n);
    for (uint32_t e = 0; e < e_count; ++e)
        if (s.ctype[e] <= 1) {
            adj[ci[e]].push_back(cj[e]);
            adj[cj[e]].push_back(ci[e]);
        }
    s.ring_off.assign(n + 1, 0);
    s.ring_idx.clear();
    std::vector<uint32_t> tmp;
    for (uint32_t i = 0; i < n; ++i) {
        tmp.clear();
        for (uint32_t a : adj[i]) {
            tmp.push_back(a);
            for (uint32_t b : adj[a]) tmp.push_back(b);
        }
        std::sort(tmp.begin(), tmp.end());
        tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
        for (uint32_t t : tmp)
            if (t != i) s.ring_idx.push_back(t);
        s.ring_off[i + 1] = (uint32_t)s.ring_idx.size();
    }
}

extern "C" {

void* oracle_sim_create(int fp64, uint32_t n, const float* x, const float* v, const float* w, const float* rest_pos,
                        uint32_t e_count, const uint32_t* ci, const uint32_t* cj, const float* rest,
                        const float* comp, const uint32_t* ctype) {
    auto* h = new OracleSim;
    h->fp64 = fp64;
    if (fp64)
        sim_init(h->d, n, x, v, w, rest_pos, e_count, ci, cj, rest, comp, ctype);
    else
        sim_init(h->f, n, x, v, w, rest_pos, e_count, ci, cj, rest, comp, ctype);
    return h;
}
void oracle_sim_free(void* h) { delete (OracleSim*)h; }

void oracle_sim_set_params(void* h, const Params* p) {
    auto* s = (OracleSim*)h;
    Params q = *p;
    // xpbd_cpu.rs:402: damp = (-linear_drag_per_sec * dt_sub).exp(), evaluated once in FP32 (libm expf)
    q.damp = std::exp(-q.linear_drag_per_sec * q.dt);
    s->f.p = q;
    s->d.p = q;
}
// Runs `count` substeps. brute_force=1 uses the all-pairs collision loop of the reference.
void oracle_sim_substeps(void* h, uint32_t count, int brute_force) {
    auto* s = (OracleSim*)h;
    for (uint32_t k = 0; k < count; ++k) {
        if (s->fp64)
            s->d.substep(brute_force != 0);
        else
            s->f.substep(brute_force != 0);
    }
}
void oracle_sim_get(void* h, double* x, double* v) {
    auto* s = (OracleSim*)h;
    auto get = [&](auto& sim) {
        for (uint32_t i = 0; i < sim.n; ++i) {
            if (x) {
                x[3 * i] = (double)sim.sim_pos[i].x;
                x[3 * i + 1] = (double)sim.sim_pos[i].y;
                x[3 * i + 2] = (double)sim.sim_pos[i].z;
            }
            if (v) {
                v[3 * i] = (double)sim.vel[i].x;
                v[3 * i + 1] = (double)sim.vel[i].y;
                v[3 * i + 2] = (double)sim.vel[i].z;
            }
        }
    };
    if (s->fp64) get(s->d); else get(s->f);
}
void oracle_sim_set_state(void* h, const float* x, const float* v) {
    auto* s = (OracleSim*)h;
    auto set = [&](auto& sim) {
        using VT = typename std::remove_reference<decltype(sim.sim_pos[0])>::type;
        using T = decltype(VT{}.x);
        for (uint32_t i = 0; i < sim.n; ++i) {
            if (x) sim.sim_pos[i] = VT{(T)x[3 * i], (T)x[3 * i + 1], (T)x[3 * i + 2]};
            if (v) sim.vel[i] = VT{(T)v[3 * i], (T)v[3 * i + 1], (T)v[3 * i + 2]};
        }
    };
    if (s->fp64) set(s->d); else set(s->f);
}
// Per-constraint λ (after the last substep) and the warm-start λ for the next substeps (NULL clears it).
void oracle_sim_get_lambda(void* h, double* out) {
    auto* s = (OracleSim*)h;
    if (s->fp64)
        for (size_t e = 0; e < s->d.lambda.size(); ++e) out[e] = s->d.lambda[e];
    else
        for (size_t e = 0; e < s->f.lambda.size(); ++e) out[e] = (double)s->f.lambda[e];
}
// Positions the next substep's prediction step would produce (state unchanged).
void oracle_sim_predicted(void* h, double* x) {
    auto* s = (OracleSim*)h;
    auto run = [&](auto& sim) {
        for (uint32_t i = 0; i < sim.n; ++i) {
            auto pos = sim.sim_pos[i];
            if (sim.inv_mass[i] > 0) {
                auto v = sim.vel[i];
                pos = sim.predict_particle(i, sim.sim_pos[i], v);
            }
            x[3 * i] = (double)pos.x;
            x[3 * i + 1] = (double)pos.y;
            x[3 * i + 2] = (double)pos.z;
        }
    };
    if (s->fp64)
        run(s->d);
    else
        run(s->f);
}
void oracle_sim_set_warm_lambda(void* h, const float* lam) {
    auto* s = (OracleSim*)h;
    if (!lam) {
        s->f.warm_lambda.clear();
        s->d.warm_lambda.clear();
        return;
    }
    size_t e = s->f.ci.size() ? s->f.ci.size() : s->d.ci.size();
    s->f.warm_lambda.assign(lam, lam + e);
    s->d.warm_lambda.resize(e);
    for (size_t k = 0; k < e; ++k) s->d.warm_lambda[k] = lam[k];
}
// Extension convergence solve (Jacobi, per-substep λ, optional warm start from oracle_sim_set_warm_lambda).
void oracle_sim_substeps_converge(void* h, uint32_t count, uint32_t* iterations_out, uint32_t* fallback_out) {
    auto* s = (OracleSim*)h;
    for (uint32_t k = 0; k < count; ++k) {
        if (s->fp64) {
            s->d.substep_converge();
            if (iterations_out) iterations_out[k] = s->d.last_iterations;
            if (fallback_out) fallback_out[k] = s->d.last_fallback;
        } else {
            s->f.substep_converge();
            if (iterations_out) iterations_out[k] = s->f.last_iterations;
            if (fallback_out) fallback_out[k] = s->f.last_fallback;
        }
    }
}
void oracle_sim_set_batches(void* h, const uint32_t* offsets, uint32_t count) {
    auto* s = (OracleSim*)h;
    std::vector<uint32_t> b;
    if (offsets) b.assign(offsets, offsets + count + 1);
    s->f.batch_off = b;
    s->d.batch_off = b;
}
int oracle_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
double oracle_sim_strain_residual(void* h) {
    auto* s = (OracleSim*)h;
    return s->fp64 ? s->d.strain_residual() : (double)s->f.strain_residual();
}
uint64_t oracle_sim_collision_pairs_last(void* h) {
    auto* s = (OracleSim*)h;
    return s->fp64 ? s->d.collision_pairs_last : s->f.collision_pairs_last;
}
// Reference self_collision_resolve on its own (xpbd_cpu.rs:67-137), FP32, in place.
void oracle_self_collision_resolve(uint32_t n, float* x, const float* inv_mass, const float* rest_pos,
                                   float thickness, float coll_scale) {
    Sim<float> s;
    s.n = n;
    s.sim_pos.resize(n);
    s.rest_pos.resize(n);
    s.inv_mass.assign(inv_mass, inv_mass + n);
    for (uint32_t i = 0; i < n; ++i) {
        s.sim_pos[i] = Sim<float>::cvt(x, i);
        s.rest_pos[i] = Sim<float>::cvt(rest_pos, i);
    }
    s.p.thickness = thickness;
    s.p.coll_scale = coll_scale;
    s.self_collision_all_pairs(1);
    for (uint32_t i = 0; i < n; ++i) {
        x[3 * i] = s.sim_pos[i].x;
        x[3 * i + 1] = s.sim_pos[i].y;
        x[3 * i + 2] = s.sim_pos[i].z;
    }
}

// ---------------------------------------------------------------------------------------------- hash spec
void oracle_hash_keys(uint32_t n, const float* xyz, float inv_cell, uint32_t table_bits, uint32_t* keys) {
    for (uint32_t i = 0; i < n; ++i)
        keys[i] = hash_cell_key(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], inv_cell, table_bits);
}
void oracle_stable_radix_sort(uint32_t n, uint32_t* keys, uint32_t* vals, int passes) {
    std::vector<uint32_t> k(keys, keys + n), v(vals, vals + n);
    stable_radix_sort(k, v, passes);
    std::copy(k.begin(), k.end(), keys);
    std::copy(v.begin(), v.end(), vals);
}
// Collision pair list (a<b, lexicographic) of the current state of a FP32 sim under its collision filter.
// Returns the pair count; writes at most `cap` pairs (2 entries each).
uint64_t oracle_sim_collision_pairs(void* h, uint32_t* pairs, uint64_t cap) {
    auto* hs = (OracleSim*)h;
    Sim<float>& s = hs->f;
    int filter = s.p.collision == 2 ? 2 : 1;
    double cell = (double)std::max(s.p.hash_cell, s.p.thickness) * 1.001;
    std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
    auto key = [](int64_t x, int64_t y, int64_t z) {
        return ((uint64_t)(x & 0x1FFFFF) << 42) | ((uint64_t)(y & 0x1FFFFF) << 21) | (uint64_t)(z & 0x1FFFFF);
    };
    std::vector<std::array<int64_t, 3>> cc(s.n);
    for (uint32_t i = 0; i < s.n; ++i) {
        cc[i] = {(int64_t)std::floor(s.sim_pos[i].x / cell), (int64_t)std::floor(s.sim_pos[i].y / cell),
                 (int64_t)std::floor(s.sim_pos[i].z / cell)};
        cells[key(cc[i][0], cc[i][1], cc[i][2])].push_back(i);
    }
    uint64_t count = 0;
    std::vector<uint32_t> cand;
    for (uint32_t i = 0; i < s.n; ++i) {
        cand.clear();
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    auto it = cells.find(key(cc[i][0] + dx, cc[i][1] + dy, cc[i][2] + dz));
                    if (it == cells.end()) continue;
                    for (uint32_t j : it->second)
                        if (j > i) cand.push_back(j);
                }
        std::sort(cand.begin(), cand.end());
        for (uint32_t j : cand) {
            V3<float> da, db;
            if (!s.narrow_pair(i, j, filter, da, db)) continue;
            if (count < cap) {
                pairs[2 * count] = i;
                pairs[2 * count + 1] = j;
            }
            ++count;
        }
    }
    return count;
}

}  // extern "C"
