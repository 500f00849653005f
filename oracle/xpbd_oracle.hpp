// ORACLE — test infrastructure only. Nothing in the product (the bevy_xpbd_b200 package, its CUDA library or
// its headers) includes, links or calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg use it, and only as the checker.
//
// CPU restatement of the reference XPBD cloth solver of mate-h/bevy_xpbd (crate `bevy_softbody`):
//   * src/xpbd_cpu.rs      — predict, Jacobi edges + gather, colored Gauss–Seidel sweep, O(n^2) self collision,
//                            post velocity, substep drivers (each function below cites the lines it follows).
//   * src/mesh_prep.rs     — grid / welded-OBJ builders, constraint generation order, area inverse mass, pins,
//                            greedy edge coloring, neighbour CSR scatter, collision grid sizing.
//   * src/cloth_compute.rs — solver constants (:57-95).
// Templated on the scalar type: T=float is the FP32 oracle (operation order identical to the Rust source, built
// with -ffp-contract=off so no multiply-add is fused, as rustc never fuses), T=double is the FP64 accuracy
// reference used to state the error of both the FP32 oracle and the CUDA path.
//
// Pinning: the reference cannot be built here (Rust toolchain and its crates.io dependencies are absent), and it
// ships no golden vectors. The restatement is pinned by porting every known-answer and invariant test of the
// reference for this path (xpbd_cpu.rs:751-1128, cloth_compute.rs:1528-1577; tests/test_oracle_reference_tests.py)
// and by the reference's one input fixture, assets/cloth.obj (copied to tests/golden/), whose parse_welded_obj result
// is checked against the structure the reference source implies (tests/test_golden_cpu.py).
//
// Additions that have no reference counterpart (marked "extension"): per-substep λ mode, degree-averaged
// Jacobi relaxation, strain residual, the spatial-hash collision specification (prime hash, stable LSD radix
// sort, 2-ring topology filter, ground plane) and the warm-start MLP.
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace oracle {

// ---- constants: cloth_compute.rs:57-95, mesh_prep.rs:87-101 -------------------------------------------------
constexpr float JACOBI_CORRECTION_CAP = 0.28f;      // cloth_compute.rs:82
constexpr float PREDICT_MAX_SPEED = 12.0f;          // cloth_compute.rs:84
constexpr float GRAB_MAX_PULL_PER_SUBSTEP = 0.065f; // cloth_compute.rs:86
constexpr float COLLISION_APPLY_CLAMP = 0.35f;      // cloth_compute.rs:90
constexpr float DEFAULT_BEND_COMPLIANCE = 3.8f;     // mesh_prep.rs:89
constexpr float DEFAULT_STRETCH_COMPLIANCE = 2e-8f; // mesh_prep.rs:93
constexpr float DEFAULT_SKIP2_COMPLIANCE = 2.5e-8f; // mesh_prep.rs:97
constexpr float DEFAULT_CROSS_DIAG_COMPLIANCE = 6e-9f; // mesh_prep.rs:101

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <typename T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <typename T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
// glam Vec3::dot = (x*x') + (y*y') + (z*z'), length = sqrt(dot(self, self)); no fused multiply-add.
template <typename T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <typename T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}

// ============================================================================================================
// Mesh preparation (mesh_prep.rs). Always FP32 like the reference: it produces the solver's inputs.
// ============================================================================================================
using V3f = V3<float>;
struct Constraint {
    uint32_t i, j;
    float rest, comp;
};

struct Mesh {  // ClothMeshData, mesh_prep.rs:103-131 (render-only fields omitted)
    std::vector<V3f> positions;
    std::vector<uint32_t> indices;
    std::vector<uint32_t> tri_edge_neighbors;
    std::vector<float> inv_mass;
    std::vector<uint32_t> neighbor_other, neighbor_constraint_id, neighbor_offsets;
    std::vector<float> neighbor_rest_len, neighbor_compliance;
    std::vector<uint32_t> constraint_i, constraint_j;
    std::vector<float> constraint_rest_len, constraint_compliance;
    std::vector<V3f> rest_positions;
    std::vector<uint32_t> constraint_batch_offsets;
    uint32_t constraint_batch_count = 0;
    uint32_t num_particles = 0;
};

inline float dist(V3f a, V3f b) { return length(a - b); }  // mesh_prep.rs:149-151

// Greedy edge coloring, mesh_prep.rs:153-221. Process order: stable sort by (max endpoint degree desc, min(i,j),
// max(i,j)) (:172-177); each edge takes the smallest color unused at both endpoints (:183-202); result stably
// sorted by (color, original index) (:204-205); batch offsets at color changes (:210-218).
// order_by_index=true is the documented "constraint-index order" variant (no degree sort).
struct Partition {
    std::vector<uint32_t> perm;    // sorted position -> original constraint index
    std::vector<uint32_t> colors;  // per sorted constraint
    std::vector<uint32_t> offsets; // batch offsets (count + 1 entries)
};
inline Partition partition_constraints_for_gs_batches(uint32_t n_particles, const std::vector<Constraint>& cons,
                                                      bool order_by_index = false) {
    Partition out;
    const size_t e_count = cons.size();
    if (e_count == 0) {
        out.offsets = {0, 0};
        return out;
    }
    std::vector<uint32_t> deg(n_particles, 0);
    for (auto& c : cons) {
        deg[c.i] += 1;
        deg[c.j] += 1;
    }
    std::vector<size_t> process_order(e_count);
    for (size_t e = 0; e < e_count; ++e) process_order[e] = e;
    if (!order_by_index) {
        std::stable_sort(process_order.begin(), process_order.end(), [&](size_t a, size_t b) {
            const auto& ca = cons[a];
            const auto& cb = cons[b];
            uint32_t da = std::max(deg[ca.i], deg[ca.j]);
            uint32_t db = std::max(deg[cb.i], deg[cb.j]);
            if (da != db) return da > db;  // Reverse(d)
            uint32_t mina = std::min(ca.i, ca.j), minb = std::min(cb.i, cb.j);
            if (mina != minb) return mina < minb;
            return std::max(ca.i, ca.j) < std::max(cb.i, cb.j);
        });
    }
    std::vector<uint32_t> color_of_edge(e_count, 0);
    std::vector<std::vector<uint32_t>> occupied(n_particles);
    std::unordered_set<uint32_t> forb;
    for (size_t e : process_order) {
        uint32_t i = cons[e].i, j = cons[e].j;
        forb.clear();
        for (uint32_t c : occupied[i]) forb.insert(c);
        for (uint32_t c : occupied[j]) forb.insert(c);
        uint32_t c = 0;
        while (forb.count(c)) c += 1;
        color_of_edge[e] = c;
        occupied[i].push_back(c);
        occupied[j].push_back(c);
    }
    std::vector<size_t> order(e_count);
    for (size_t e = 0; e < e_count; ++e) order[e] = e;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (color_of_edge[a] != color_of_edge[b]) return color_of_edge[a] < color_of_edge[b];
        return a < b;
    });
    out.perm.resize(e_count);
    out.colors.resize(e_count);
    for (size_t k = 0; k < e_count; ++k) {
        out.perm[k] = (uint32_t)order[k];
        out.colors[k] = color_of_edge[order[k]];
    }
    out.offsets.push_back(0);
    for (size_t k = 1; k < e_count; ++k)
        if (out.colors[k] != out.colors[k - 1]) out.offsets.push_back((uint32_t)k);
    out.offsets.push_back((uint32_t)e_count);
    return out;
}

// Neighbour CSR, cursor scatter in (batch-sorted) constraint order, mesh_prep.rs:588-635.
struct Csr {
    std::vector<uint32_t> offsets, other, eid;
};
inline Csr build_neighbor_csr(uint32_t n, const std::vector<uint32_t>& ci, const std::vector<uint32_t>& cj) {
    Csr csr;
    csr.offsets.assign(n + 1, 0);
    std::vector<uint32_t> counts(n, 0);
    for (size_t e = 0; e < ci.size(); ++e) {
        counts[ci[e]] += 1;
        counts[cj[e]] += 1;
    }
    for (uint32_t i = 0; i < n; ++i) csr.offsets[i + 1] = csr.offsets[i] + counts[i];
    size_t nn = csr.offsets[n];
    csr.other.assign(nn, 0);
    csr.eid.assign(nn, 0);
    std::vector<uint32_t> cursors(csr.offsets.begin(), csr.offsets.begin() + n);
    for (size_t e = 0; e < ci.size(); ++e) {
        uint32_t i = ci[e], j = cj[e];
        uint32_t pi = cursors[i]++;
        csr.other[pi] = j;
        csr.eid[pi] = (uint32_t)e;
        uint32_t pj = cursors[j]++;
        csr.other[pj] = i;
        csr.eid[pj] = (uint32_t)e;
    }
    return csr;
}

// find_tri_neighbors, mesh_prep.rs:661-695 (Rust sort_by is stable).
inline std::vector<uint32_t> find_tri_neighbors(const std::vector<uint32_t>& indices) {
    size_t num_tris = indices.size() / 3;
    struct Edge {
        uint32_t id0, id1, edge_nr;
    };
    std::vector<Edge> edges;
    edges.reserve(num_tris * 3);
    for (size_t i = 0; i < num_tris; ++i)
        for (uint32_t j = 0; j < 3; ++j) {
            uint32_t a = indices[3 * i + j], b = indices[3 * i + (j + 1) % 3];
            edges.push_back({std::min(a, b), std::max(a, b), (uint32_t)(3 * i + j)});
        }
    std::stable_sort(edges.begin(), edges.end(), [](const Edge& a, const Edge& b) {
        if (a.id0 != b.id0) return a.id0 < b.id0;
        return a.id1 < b.id1;
    });
    std::vector<uint32_t> nb(3 * num_tris, 0xFFFFFFFFu);
    for (size_t i = 0; i + 1 < edges.size(); ++i) {
        const Edge& e0 = edges[i];
        const Edge& e1 = edges[i + 1];
        if (e0.id0 == e1.id0 && e0.id1 == e1.id1) {
            nb[e0.edge_nr] = e1.edge_nr;
            nb[e1.edge_nr] = e0.edge_nr;
        }
    }
    return nb;
}

struct Pair3 {
    uint32_t a, b;
    float rest;
};
// unique_edges_and_rests, mesh_prep.rs:697-722.
inline std::vector<Pair3> unique_edges_and_rests(const std::vector<uint32_t>& idx, const std::vector<V3f>& pos,
                                                 const std::vector<uint32_t>& nb) {
    std::set<std::pair<uint32_t, uint32_t>> seen;
    std::vector<Pair3> out;
    size_t num_tris = idx.size() / 3;
    for (size_t i = 0; i < num_tris; ++i)
        for (uint32_t j = 0; j < 3; ++j) {
            uint32_t id0 = idx[3 * i + j], id1 = idx[3 * i + (j + 1) % 3];
            uint32_t n = nb[3 * i + j];
            if (n != 0xFFFFFFFFu && id0 >= id1) continue;
            uint32_t a = std::min(id0, id1), b = std::max(id0, id1);
            if (seen.insert({a, b}).second) out.push_back({a, b, dist(pos[a], pos[b])});
        }
    return out;
}
// bending_pairs, mesh_prep.rs:724-747.
inline std::vector<Pair3> bending_pairs(const std::vector<uint32_t>& idx, const std::vector<uint32_t>& nb,
                                        const std::vector<V3f>& pos) {
    std::set<std::pair<uint32_t, uint32_t>> seen;
    std::vector<Pair3> out;
    size_t num_tris = idx.size() / 3;
    for (size_t i = 0; i < num_tris; ++i)
        for (uint32_t j = 0; j < 3; ++j) {
            uint32_t n = nb[3 * i + j];
            if (n == 0xFFFFFFFFu) continue;
            uint32_t id2 = idx[3 * i + (j + 2) % 3];
            uint32_t ni = n / 3, nj = n % 3;
            uint32_t id3 = idx[3 * ni + (nj + 2) % 3];
            uint32_t a = std::min(id2, id3), b = std::max(id2, id3);
            if (seen.insert({a, b}).second) out.push_back({a, b, dist(pos[a], pos[b])});
        }
    return out;
}

// finalize_cloth_mesh, mesh_prep.rs:532-659.
inline Mesh finalize_cloth_mesh(std::vector<V3f> positions, std::vector<uint32_t> indices,
                                const std::vector<Constraint>& extras) {
    Mesh m;
    size_t n = positions.size();
    size_t num_tris = indices.size() / 3;
    m.inv_mass.assign(n, 0.0f);
    for (size_t t = 0; t < num_tris; ++t) {  // :542-554
        uint32_t id0 = indices[3 * t], id1 = indices[3 * t + 1], id2 = indices[3 * t + 2];
        V3f e0 = positions[id1] - positions[id0];
        V3f e1 = positions[id2] - positions[id0];
        V3f c = cross(e0, e1);
        float a = 0.5f * length(c);
        float p_inv = a > 0.0f ? 1.0f / a / 3.0f : 0.0f;
        m.inv_mass[id0] += p_inv;
        m.inv_mass[id1] += p_inv;
        m.inv_mass[id2] += p_inv;
    }
    m.tri_edge_neighbors = find_tri_neighbors(indices);
    float max_y = -INFINITY;  // :558-568
    for (auto& p : positions) max_y = std::max(max_y, p.y);
    const float eps = 1e-5f;
    for (size_t i = 0; i < n; ++i)
        if (positions[i].y >= max_y - eps) m.inv_mass[i] = 0.0f;
    m.rest_positions = positions;
    auto edge_pairs = unique_edges_and_rests(indices, positions, m.tri_edge_neighbors);
    auto bend_pairs = bending_pairs(indices, m.tri_edge_neighbors, positions);
    std::vector<Constraint> cons;  // :575-582
    for (auto& p : edge_pairs) cons.push_back({p.a, p.b, p.rest, DEFAULT_STRETCH_COMPLIANCE});
    for (auto& p : bend_pairs) cons.push_back({p.a, p.b, p.rest, DEFAULT_BEND_COMPLIANCE});
    cons.insert(cons.end(), extras.begin(), extras.end());
    Partition part = partition_constraints_for_gs_batches((uint32_t)n, cons);
    for (uint32_t k : part.perm) {
        m.constraint_i.push_back(cons[k].i);
        m.constraint_j.push_back(cons[k].j);
        m.constraint_rest_len.push_back(cons[k].rest);
        m.constraint_compliance.push_back(cons[k].comp);
    }
    m.constraint_batch_offsets = part.offsets;
    m.constraint_batch_count = (uint32_t)(part.offsets.size() - 1);
    Csr csr = build_neighbor_csr((uint32_t)n, m.constraint_i, m.constraint_j);
    m.neighbor_offsets = csr.offsets;
    m.neighbor_other = csr.other;
    m.neighbor_constraint_id = csr.eid;
    for (uint32_t e : csr.eid) {
        m.neighbor_rest_len.push_back(m.constraint_rest_len[e]);
        m.neighbor_compliance.push_back(m.constraint_compliance[e]);
    }
    m.positions = std::move(positions);
    m.indices = std::move(indices);
    m.num_particles = (uint32_t)n;
    return m;
}

// grid_cloth_hanging, mesh_prep.rs:363-406 (+ :409-426 cross diagonals, :504-530 skip-2 braces).
inline Mesh grid_cloth_hanging(uint32_t quad_cols, uint32_t quad_rows, float cell_size) {
    uint32_t vc = quad_cols + 1, vr = quad_rows + 1;
    std::vector<V3f> pos;
    float width = (float)quad_cols * cell_size;
    float x0 = -0.5f * width;
    for (uint32_t iy = 0; iy < vr; ++iy)
        for (uint32_t ix = 0; ix < vc; ++ix) pos.push_back({x0 + (float)ix * cell_size, (float)iy * cell_size, 0.0f});
    std::vector<uint32_t> idx;
    size_t cols = vc;
    for (size_t iy = 0; iy < quad_rows; ++iy)
        for (size_t ix = 0; ix < quad_cols; ++ix) {
            uint32_t i0 = (uint32_t)(iy * cols + ix), i1 = i0 + 1, i2 = (uint32_t)(i0 + cols), i3 = i2 + 1;
            idx.insert(idx.end(), {i0, i1, i2, i1, i3, i2});
        }
    std::vector<Constraint> extras;
    for (size_t iy = 0; iy < vr; ++iy)  // grid_skip_two_distance_constraints, rows then columns
        for (size_t ix = 0; ix + 2 < vc; ++ix) {
            uint32_t i = (uint32_t)(iy * cols + ix), j = i + 2;
            extras.push_back({i, j, dist(pos[i], pos[j]), DEFAULT_SKIP2_COMPLIANCE});
        }
    for (size_t iy = 0; iy + 2 < vr; ++iy)
        for (size_t ix = 0; ix < vc; ++ix) {
            uint32_t i = (uint32_t)(iy * cols + ix), j = (uint32_t)((iy + 2) * cols + ix);
            extras.push_back({i, j, dist(pos[i], pos[j]), DEFAULT_SKIP2_COMPLIANCE});
        }
    for (size_t iy = 0; iy < quad_rows; ++iy)  // grid_quad_cross_diagonal_constraints
        for (size_t ix = 0; ix < quad_cols; ++ix) {
            size_t i0 = iy * cols + ix, i3 = (iy + 1) * cols + ix + 1;
            extras.push_back({(uint32_t)std::min(i0, i3), (uint32_t)std::max(i0, i3), dist(pos[i0], pos[i3]),
                              DEFAULT_CROSS_DIAG_COMPLIANCE});
        }
    return finalize_cloth_mesh(std::move(pos), std::move(idx), extras);
}

// dedup_sorted_coords, mesh_prep.rs:429-439.
inline void dedup_sorted_coords(std::vector<float>& v, float eps) {
    std::stable_sort(v.begin(), v.end(), [](float a, float b) { return a < b; });
    size_t w = 0;
    for (size_t r = 0; r < v.size(); ++r)
        if (w == 0 || std::fabs(v[r] - v[w - 1]) > eps) v[w++] = v[r];
    v.resize(w);
}
// axis_aligned_grid_skip_two_distance_constraints, mesh_prep.rs:444-501. Returns false for "None".
inline bool axis_aligned_grid_skip_two(const std::vector<V3f>& pos, std::vector<Constraint>& out) {
    const float EPS = 2e-4f;
    if (pos.empty()) return false;
    std::vector<float> xs, ys;
    for (auto& p : pos) {
        xs.push_back(p.x);
        ys.push_back(p.y);
    }
    dedup_sorted_coords(xs, EPS);
    dedup_sorted_coords(ys, EPS);
    size_t cols = xs.size(), rows = ys.size();
    if (cols < 3 || rows < 3 || cols * rows != pos.size()) return false;
    std::vector<int64_t> grid(cols * rows, -1);
    for (size_t pid = 0; pid < pos.size(); ++pid) {
        long ix = -1, iy = -1;
        for (size_t k = 0; k < cols; ++k)
            if (std::fabs(xs[k] - pos[pid].x) <= EPS) { ix = (long)k; break; }
        for (size_t k = 0; k < rows; ++k)
            if (std::fabs(ys[k] - pos[pid].y) <= EPS) { iy = (long)k; break; }
        if (ix < 0 || iy < 0) return false;
        size_t slot = (size_t)iy * cols + (size_t)ix;
        if (grid[slot] >= 0) return false;
        grid[slot] = (int64_t)pid;
    }
    for (auto g : grid)
        if (g < 0) return false;
    auto at = [&](size_t ix, size_t iy) { return (uint32_t)grid[iy * cols + ix]; };
    for (size_t iy = 0; iy < rows; ++iy)
        for (size_t ix = 0; ix + 2 < cols; ++ix) {
            uint32_t i = at(ix, iy), j = at(ix + 2, iy);
            out.push_back({std::min(i, j), std::max(i, j), dist(pos[i], pos[j]), DEFAULT_SKIP2_COMPLIANCE});
        }
    for (size_t iy = 0; iy + 2 < rows; ++iy)
        for (size_t ix = 0; ix < cols; ++ix) {
            uint32_t i = at(ix, iy), j = at(ix, iy + 2);
            out.push_back({std::min(i, j), std::max(i, j), dist(pos[i], pos[j]), DEFAULT_SKIP2_COMPLIANCE});
        }
    return true;
}

// parse_welded_obj, mesh_prep.rs:223-357 (normals/uvs are render-only and not kept).
// Rust's str::parse::<usize>: an optional '+', then at least one decimal digit; overflow is an error.
inline bool parse_usize(const std::string& s, size_t& out) {
    size_t k = (!s.empty() && s[0] == '+') ? 1 : 0;
    if (k == s.size()) return false;
    size_t v = 0;
    for (; k < s.size(); ++k) {
        const char ch = s[k];
        if (ch < '0' || ch > '9') return false;
        const size_t d = (size_t)(ch - '0');
        if (v > (SIZE_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    out = v;
    return true;
}
inline bool parse_f32(const std::string& s, float& out) {
    if (s.empty()) return false;
    char* end = nullptr;
    float v = std::strtof(s.c_str(), &end);
    if (end == s.c_str() || *end != '\0') return false;
    out = v;
    return true;
}
inline Mesh parse_welded_obj(const std::string& text) {
    std::vector<std::array<float, 3>> vp;
    std::vector<std::vector<std::string>> faces;
    size_t start = 0;
    while (start <= text.size()) {
        size_t nl = text.find('\n', start);
        std::string line = text.substr(start, nl == std::string::npos ? std::string::npos : nl - start);
        start = (nl == std::string::npos) ? text.size() + 1 : nl + 1;
        // trim
        size_t a = line.find_first_not_of(" \t\r\f\v");
        if (a == std::string::npos) continue;
        size_t b = line.find_last_not_of(" \t\r\f\v");
        line = line.substr(a, b - a + 1);
        if (line.empty() || line[0] == '#') continue;
        std::vector<std::string> parts;
        size_t p = 0;
        while (p < line.size()) {
            while (p < line.size() && isspace((unsigned char)line[p])) ++p;
            size_t q = p;
            while (q < line.size() && !isspace((unsigned char)line[q])) ++q;
            if (q > p) parts.push_back(line.substr(p, q - p));
            p = q;
        }
        if (parts.empty()) continue;
        if (parts[0] == "v") {
            float c[3] = {0, 0, 0};
            for (int k = 0; k < 3; ++k) {
                float v;
                if ((size_t)(k + 1) < parts.size() && parse_f32(parts[k + 1], v)) c[k] = v;
            }
            vp.push_back({c[0], c[1], c[2]});
        } else if (parts[0] == "f") {
            faces.emplace_back(parts.begin() + 1, parts.end());
        }
    }
    std::unordered_map<std::string, uint32_t> cache;
    std::vector<V3f> positions;
    std::vector<uint32_t> indices;
    std::vector<std::pair<uint32_t, uint32_t>> quad_cross;
    auto corner_index = [&](const std::string& fs) -> uint32_t {
        auto it = cache.find(fs);
        if (it != cache.end()) return it->second;
        uint32_t idx = (uint32_t)positions.size();
        cache[fs] = idx;
        std::string first = fs.substr(0, fs.find('/'));
        size_t vi = 1;
        size_t parsed;
        if (parse_usize(first, parsed)) vi = parsed;
        vi = vi == 0 ? 0 : vi - 1;  // saturating_sub(1)
        if (vi < vp.size())
            positions.push_back({vp[vi][0], vp[vi][1], vp[vi][2]});
        else
            positions.push_back({0.0f, 0.0f, 0.0f});
        return idx;
    };
    for (auto& face : faces) {
        if (face.size() < 3) continue;
        if (face.size() == 4) {
            uint32_t v0 = corner_index(face[0]), v1 = corner_index(face[1]);
            uint32_t v2 = corner_index(face[2]), v3 = corner_index(face[3]);
            indices.insert(indices.end(), {v0, v1, v2, v0, v2, v3});
            quad_cross.push_back({std::min(v1, v3), std::max(v1, v3)});
            continue;
        }
        uint32_t c0 = corner_index(face[0]);
        for (size_t i = 1; i + 1 < face.size(); ++i) {
            indices.push_back(c0);
            indices.push_back(corner_index(face[i]));
            indices.push_back(corner_index(face[i + 1]));
        }
    }
    std::vector<Constraint> extras;
    std::vector<Constraint> skip2;
    if (axis_aligned_grid_skip_two(positions, skip2)) extras = skip2;
    for (auto& qc : quad_cross)
        extras.push_back({qc.first, qc.second, dist(positions[qc.first], positions[qc.second]),
                          DEFAULT_CROSS_DIAG_COMPLIANCE});
    return finalize_cloth_mesh(std::move(positions), std::move(indices), extras);
}

// ============================================================================================================
// Solver state and substep (xpbd_cpu.rs), templated on T.
// ============================================================================================================
struct Params {  // XpbdCpuTimeStepParams, xpbd_cpu.rs:11-26, plus the extension modes
    float dt, inv_dt, jacobi_omega;
    uint32_t inner_iterations;
    float gravity[3];
    int32_t grab_idx;
    uint32_t grab_active;
    float grab_target[3];
    float grab_stiffness;
    float linear_drag_per_sec;
    uint32_t solver;       // 0 Jacobi (solver-jacobi), 1 colored Gauss-Seidel (solver-gauss-seidel)
    uint32_t relaxation;   // 0 ω·acc (reference), 1 extension: (ω·acc)/degree
    uint32_t lambda_mode;  // 0 λ cleared every inner iteration (reference :267), 1 extension: once per substep
    uint32_t collision;    // 0 none, 1 reference O(n^2) (:67-137), 2 extension: hashed with 2-ring filter
    float thickness, coll_scale;
    float hash_cell;
    uint32_t ground_enabled;
    float ground_y;
    float damp;            // exp(-k·dt) evaluated once on the host (xpbd_cpu.rs:402)
    float tolerance;       // extension: stop when the pre-update residual max|C+α̃λ|/rest <= tolerance (0 = off)
    uint32_t warm_start;   // extension: 1 = start from the given λ0 (warm_lambda) when it lowers the residual
    float wind[3];         // extension: wind velocity; after gravity v += (wind - v) * (wind_drag * dt)
    float wind_drag;       // 0 = no wind
};

template <typename T>
struct Sim {
    using V = V3<T>;
    uint32_t n = 0;
    std::vector<V> sim_pos, prev_pos, vel, jac_a, jac_b, rest_pos;
    std::vector<T> inv_mass;
    std::vector<uint32_t> ci, cj, ctype;
    std::vector<T> rest, comp;
    std::vector<uint32_t> nb_off, nb_other, nb_eid;
    std::vector<uint32_t> batch_off;  // optional color batches: lets the OpenMP build sweep a batch in parallel
    std::vector<T> lambda, delta_lambda;
    std::vector<T> warm_lambda;  // extension: initial λ for the per-substep mode (empty → zeros)
    // 2-ring topology lists (extension collision filter): sorted, per vertex
    std::vector<uint32_t> ring_off, ring_idx;
    Params p{};
    uint64_t collision_pairs_last = 0;
    uint32_t last_iterations = 0;  // convergence solve: update passes of the last substep
    uint32_t last_fallback = 0;    // convergence solve: 1 if the warm start was rejected in the last substep

    static V cvt(const float* a, size_t i) { return {(T)a[3 * i], (T)a[3 * i + 1], (T)a[3 * i + 2]}; }

    // clamp_correction, xpbd_cpu.rs:28-36
    static V clamp_correction(V dx) {
        T ml = length(dx);
        T cap = (T)JACOBI_CORRECTION_CAP;
        if (ml > cap && ml > (T)0) return dx * (cap / ml);
        return dx;
    }

    // predict_particle, xpbd_cpu.rs:38-65
    V predict_particle(uint32_t i, V sim, V& vel_io) const {
        V v = vel_io;
        V g = {(T)p.gravity[0], (T)p.gravity[1], (T)p.gravity[2]};
        T dt = (T)p.dt;
        v = v + g * dt;
        if (p.wind_drag > 0.0f) {  // extension: wind (no reference counterpart)
            V wv = {(T)p.wind[0], (T)p.wind[1], (T)p.wind[2]};
            v = v + (wv - v) * (T)(p.wind_drag * p.dt);
        }
        T speed = length(v);
        T max_v = (T)PREDICT_MAX_SPEED;
        if (speed > max_v && speed > (T)0) v = v * (max_v / speed);
        V pos = sim + v * dt;
        if (p.grab_active && (int32_t)i == p.grab_idx) {
            V tgt = {(T)p.grab_target[0], (T)p.grab_target[1], (T)p.grab_target[2]};
            V pull = (tgt - pos) * (T)p.grab_stiffness;
            T pl = length(pull);
            T gmax = (T)GRAB_MAX_PULL_PER_SUBSTEP;
            if (pl > gmax && pl > (T)0) pull = pull * (gmax / pl);
            pos = pos + pull;
        }
        vel_io = v;
        return pos;
    }

    // jacobi_edges_pass, xpbd_cpu.rs:139-184
    void jacobi_edges_pass(const std::vector<V>& jin, T inv_dt_sq) {
#pragma omp parallel for schedule(static)
        for (size_t e = 0; e < ci.size(); ++e) {
            uint32_t i = ci[e], j = cj[e];
            T w_i = inv_mass[i], w_j = inv_mass[j];
            if (w_j <= (T)0 && w_i <= (T)0) { delta_lambda[e] = 0; continue; }
            V gv = jin[i] - jin[j];
            T len = length(gv);
            if (len < (T)1e-8f) { delta_lambda[e] = 0; continue; }
            T c = len - rest[e];
            T alpha_t = comp[e] * inv_dt_sq;
            T wsum = w_i + w_j + alpha_t;
            if (wsum < (T)1e-8f) { delta_lambda[e] = 0; continue; }
            T lam = lambda[e];
            T dlam = (-c - alpha_t * lam) / wsum;
            delta_lambda[e] = dlam;
            lambda[e] = lam + dlam;
        }
    }

    // jacobi_gather_particle, xpbd_cpu.rs:186-226 (relaxation 1 divides ω·acc by the CSR row length)
    V jacobi_gather_particle(uint32_t i, const std::vector<V>& jin) const {
        T w_i = inv_mass[i];
        if (w_i <= (T)0) return jin[i];
        V p_i = jin[i];
        V acc = {0, 0, 0};
        uint32_t s = nb_off[i], en = nb_off[i + 1];
        for (uint32_t k = s; k < en; ++k) {
            uint32_t j = nb_other[k];
            T w_j = inv_mass[j];
            if (w_j <= (T)0 && w_i <= (T)0) continue;
            V gv = p_i - jin[j];
            T len = length(gv);
            if (len < (T)1e-8f) continue;
            gv = gv / len;
            T dlam = delta_lambda[nb_eid[k]];
            acc = acc + (gv * w_i) * dlam;
        }
        V delta = (T)p.jacobi_omega * acc;
        if (p.relaxation == 1 && en > s) delta = delta / (T)(en - s);
        delta = clamp_correction(delta);
        return p_i + delta;
    }

    void predict_all() {  // xpbd_cpu.rs:251-260
#pragma omp parallel for schedule(static)
        for (uint32_t i = 0; i < n; ++i) {
            if (inv_mass[i] <= (T)0) { prev_pos[i] = sim_pos[i]; continue; }
            V v = vel[i];
            V np = predict_particle(i, sim_pos[i], v);
            prev_pos[i] = sim_pos[i];
            sim_pos[i] = np;
            vel[i] = v;
        }
    }

    void begin_substep_lambda() {
        std::fill(lambda.begin(), lambda.end(), (T)0);
        std::fill(delta_lambda.begin(), delta_lambda.end(), (T)0);
        if (p.lambda_mode == 1 && warm_lambda.size() == lambda.size())
            for (size_t e = 0; e < lambda.size(); ++e) lambda[e] = warm_lambda[e];
    }

    // xpbd_substep_integrate (solver-jacobi), xpbd_cpu.rs:228-310
    void integrate_jacobi() {
        T inv_dt_sq = (T)p.inv_dt * (T)p.inv_dt;
        predict_all();
        for (uint32_t i = 0; i < n; ++i) jac_b[i] = sim_pos[i];
        begin_substep_lambda();
        for (uint32_t k = 0; k < p.inner_iterations; ++k) {
            if (p.lambda_mode == 0) {
                std::fill(lambda.begin(), lambda.end(), (T)0);
                std::fill(delta_lambda.begin(), delta_lambda.end(), (T)0);
            }
            const std::vector<V>& rd = (k % 2 == 0) ? jac_b : jac_a;
            std::vector<V>& wr = (k % 2 == 0) ? jac_a : jac_b;
            jacobi_edges_pass(rd, inv_dt_sq);
#pragma omp parallel for schedule(static)
            for (uint32_t i = 0; i < n; ++i) wr[i] = jacobi_gather_particle(i, rd);
        }
        const std::vector<V>& fin = (p.inner_iterations % 2 == 0) ? jac_b : jac_a;
        for (uint32_t i = 0; i < n; ++i) sim_pos[i] = fin[i];
    }

    // xpbd_substep_integrate (solver-gauss-seidel), xpbd_cpu.rs:312-391
    void integrate_gs() {
        predict_all();
        std::vector<V>& jw = jac_a;
        for (uint32_t i = 0; i < n; ++i) jw[i] = sim_pos[i];
        begin_substep_lambda();
        T omega = (T)p.jacobi_omega;
        T inv_dt_sq = (T)p.inv_dt * (T)p.inv_dt;
        auto solve = [&](size_t e) {
                uint32_t i = ci[e], j = cj[e];
                T w_i = inv_mass[i], w_j = inv_mass[j];
                if (w_j <= (T)0 && w_i <= (T)0) return;
                V p_i = jw[i], p_j = jw[j];
                V gv = p_i - p_j;
                T len = length(gv);
                if (len < (T)1e-8f) return;
                gv = gv / len;
                T c = len - rest[e];
                T alpha_t = comp[e] * inv_dt_sq;
                T wsum = w_i + w_j + alpha_t;
                if (wsum < (T)1e-8f) return;
                T lam = lambda[e];
                T dlam = (-c - alpha_t * lam) / wsum;
                lambda[e] = lam + dlam;
                V dx_i = clamp_correction(((omega * gv) * w_i) * dlam);
                V dx_j = clamp_correction(-(((omega * gv) * w_j) * dlam));
                if (w_i > (T)0) jw[i] = p_i + dx_i;
                if (w_j > (T)0) jw[j] = p_j + dx_j;
        };
        for (uint32_t k = 0; k < p.inner_iterations; ++k) {
            if (p.lambda_mode == 0) std::fill(lambda.begin(), lambda.end(), (T)0);
            if (batch_off.size() >= 2) {
                // a batch's constraints share no particle: any order (or parallel) gives the sequential result
                for (size_t b = 0; b + 1 < batch_off.size(); ++b) {
                    const long e0 = batch_off[b], e1 = batch_off[b + 1];
#pragma omp parallel for schedule(static)
                    for (long e = e0; e < e1; ++e) solve((size_t)e);
                }
            } else {
                for (size_t e = 0; e < ci.size(); ++e) solve(e);
            }
        }
        for (uint32_t i = 0; i < n; ++i) sim_pos[i] = jw[i];
    }

    // Extension: residual of constraint e at positions `pos` with multiplier `lam`: |C + α̃λ| / rest.
    T constraint_residual(const std::vector<V>& pos, size_t e, T lam, T inv_dt_sq) const {
        T len = length(pos[ci[e]] - pos[cj[e]]);
        T c = len - rest[e];
        T alpha_t = comp[e] * inv_dt_sq;
        return std::fabs(c + alpha_t * lam) / rest[e];
    }
    // Extension: the gather of jacobi_gather_particle with Δλ replaced by `dl` (per constraint), from `src`.
    void gather_with(const std::vector<V>& src, const std::vector<T>& dl, std::vector<V>& dst) {
        std::vector<T> saved = delta_lambda;
        delta_lambda = dl;
        for (uint32_t i = 0; i < n; ++i) dst[i] = jacobi_gather_particle(i, src);
        delta_lambda = saved;
    }
    // Extension: Jacobi substep (per-substep λ) iterating until the pre-update residual <= tolerance, at most
    // p.inner_iterations passes. Warm start: positions move by the gather of λ0 (warm_lambda) and λ starts at λ0 —
    // kept only if the resulting residual is not above the plain start's (otherwise plain: λ = 0).
    void substep_converge() {
        T inv_dt_sq = (T)p.inv_dt * (T)p.inv_dt;
        predict_all();
        std::vector<V>& start = jac_b;
        for (uint32_t i = 0; i < n; ++i) start[i] = sim_pos[i];
        std::fill(lambda.begin(), lambda.end(), (T)0);
        last_fallback = 0;
        if (p.warm_start && warm_lambda.size() == lambda.size()) {
            T plain = 0;
            for (size_t e = 0; e < ci.size(); ++e)
                if (!(inv_mass[ci[e]] <= (T)0 && inv_mass[cj[e]] <= (T)0))
                    plain = std::max(plain, constraint_residual(start, e, (T)0, inv_dt_sq));
            gather_with(start, warm_lambda, jac_a);
            T warm = 0;
            for (size_t e = 0; e < ci.size(); ++e)
                if (!(inv_mass[ci[e]] <= (T)0 && inv_mass[cj[e]] <= (T)0))
                    warm = std::max(warm, constraint_residual(jac_a, e, warm_lambda[e], inv_dt_sq));
            if (warm <= plain) {
                for (uint32_t i = 0; i < n; ++i) start[i] = jac_a[i];
                lambda = warm_lambda;
            } else {
                last_fallback = 1;
            }
        }
        uint32_t it = 0;
        std::vector<V>* cur = &jac_b;
        std::vector<V>* nxt = &jac_a;
        while (it < p.inner_iterations) {
            T res = 0;
            for (size_t e = 0; e < ci.size(); ++e)
                if (!(inv_mass[ci[e]] <= (T)0 && inv_mass[cj[e]] <= (T)0))
                    res = std::max(res, constraint_residual(*cur, e, lambda[e], inv_dt_sq));
            jacobi_edges_pass(*cur, inv_dt_sq);
            for (uint32_t i = 0; i < n; ++i) (*nxt)[i] = jacobi_gather_particle(i, *cur);
            std::swap(cur, nxt);
            ++it;
            if (res <= (T)p.tolerance) break;
        }
        last_iterations = it;
        for (uint32_t i = 0; i < n; ++i) sim_pos[i] = (*cur)[i];
        post_velocity();
    }

    // Narrow phase of one pair (a<b), xpbd_cpu.rs:84-121. filter 1: reference rest-distance test (:94-100);
    // filter 2 (extension): skip b within the 2-ring of a. Returns false when the pair is skipped.
    bool narrow_pair(uint32_t a, uint32_t b, int filter, V& da, V& db) const {
        if (inv_mass[a] <= (T)0 && inv_mass[b] <= (T)0) return false;
        T thickness = (T)p.thickness;
        T thickness_sq = thickness * thickness;
        V d = sim_pos[b] - sim_pos[a];
        T dist2 = dot(d, d);
        if (dist2 > thickness_sq || dist2 < (T)1e-18f) return false;
        V rest_d = rest_pos[b] - rest_pos[a];
        T rest2 = dot(rest_d, rest_d);
        if (filter == 1) {
            if (dist2 > rest2) return false;
        } else {
            if (in_ring(a, b)) return false;
        }
        T min_d = thickness;
        if (rest2 < thickness_sq) min_d = std::sqrt(rest2);
        T dist = std::sqrt(dist2);
        T corr = (min_d - dist) * (T)0.5f * (T)p.coll_scale;
        if (corr <= (T)0) return false;
        d = (d / dist) * corr;
        T w_i = inv_mass[a], w_j = inv_mass[b];
        T inv_w = (T)1 / std::max(w_i + w_j, (T)1e-8f);
        da = (-d * w_i) * inv_w;
        db = (d * w_j) * inv_w;
        return true;
    }
    bool in_ring(uint32_t a, uint32_t b) const {
        if (ring_off.empty()) return false;
        auto first = ring_idx.begin() + ring_off[a];
        auto last = ring_idx.begin() + ring_off[a + 1];
        return std::binary_search(first, last, b);
    }

    // self_collision_resolve, xpbd_cpu.rs:67-137: all pairs i<j, contributions summed per particle in increasing
    // partner index, then clamped per component and applied to unpinned particles.
    void self_collision_all_pairs(int filter) {
        std::vector<V> accum(n, V{0, 0, 0});
        uint64_t pairs = 0;
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t j = i + 1; j < n; ++j) {
                V di, dj;
                if (!narrow_pair(i, j, filter, di, dj)) continue;
                ++pairs;
                if (inv_mass[i] > (T)0) accum[i] = accum[i] + di;
                if (inv_mass[j] > (T)0) accum[j] = accum[j] + dj;
            }
        apply_collision(accum);
        collision_pairs_last = pairs;
    }
    // Same result as self_collision_all_pairs, candidates from a uniform cell grid (cell >= thickness) so large
    // sheets finish in seconds; partners are visited in increasing index order exactly as the all-pairs loop.
    void self_collision_grid(int filter) {
        // slightly enlarged cell: a pair within `thickness` is then always in adjacent cells despite rounding
        double cell = (double)std::max(p.hash_cell, p.thickness) * 1.001;
        std::unordered_map<uint64_t, std::vector<uint32_t>> cells;
        auto key = [](int64_t x, int64_t y, int64_t z) {
            return ((uint64_t)(x & 0x1FFFFF) << 42) | ((uint64_t)(y & 0x1FFFFF) << 21) | (uint64_t)(z & 0x1FFFFF);
        };
        std::vector<std::array<int64_t, 3>> cc(n);
        for (uint32_t i = 0; i < n; ++i) {
            cc[i] = {(int64_t)std::floor((double)sim_pos[i].x / cell), (int64_t)std::floor((double)sim_pos[i].y / cell),
                     (int64_t)std::floor((double)sim_pos[i].z / cell)};
            cells[key(cc[i][0], cc[i][1], cc[i][2])].push_back(i);
        }
        std::vector<V> accum(n, V{0, 0, 0});
        uint64_t pairs = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : pairs)
        for (uint32_t i = 0; i < n; ++i) {
            std::vector<uint32_t> cand;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        auto it = cells.find(key(cc[i][0] + dx, cc[i][1] + dy, cc[i][2] + dz));
                        if (it == cells.end()) continue;
                        for (uint32_t j : it->second)
                            if (j != i) cand.push_back(j);
                    }
            std::sort(cand.begin(), cand.end());
            for (uint32_t j : cand) {
                uint32_t a = std::min(i, j), b = std::max(i, j);
                V da, db;
                if (!narrow_pair(a, b, filter, da, db)) continue;
                if (i < j) ++pairs;
                if (inv_mass[i] > (T)0) accum[i] = accum[i] + (i == a ? da : db);
            }
        }
        apply_collision(accum);
        collision_pairs_last = pairs;
    }
    void apply_collision(const std::vector<V>& accum) {  // xpbd_cpu.rs:125-136
        T max_d = (T)COLLISION_APPLY_CLAMP;
        for (uint32_t i = 0; i < n; ++i) {
            if (inv_mass[i] <= (T)0) continue;
            V c = accum[i];
            V cl = {std::min(std::max(c.x, -max_d), max_d), std::min(std::max(c.y, -max_d), max_d),
                    std::min(std::max(c.z, -max_d), max_d)};
            sim_pos[i] = sim_pos[i] + cl;
        }
    }

    // xpbd_substep_post_velocity, xpbd_cpu.rs:393-409 (damp precomputed as exp(-k·dt)); the ground plane is an
    // extension applied to unpinned particles just before the velocity update.
    void post_velocity() {
        T damp = (T)p.damp;
        T inv_dt = (T)p.inv_dt;
        T gy = (T)p.ground_y;
#pragma omp parallel for schedule(static)
        for (uint32_t i = 0; i < n; ++i) {
            if (inv_mass[i] <= (T)0) continue;
            if (p.ground_enabled && sim_pos[i].y < gy) sim_pos[i].y = gy;
            vel[i] = ((sim_pos[i] - prev_pos[i]) * inv_dt) * damp;
        }
    }

    // xpbd_substep_no_collision / xpbd_substep_with_self_collision, xpbd_cpu.rs:411-578
    void substep(bool brute_force_collision) {
        if (p.solver == 0)
            integrate_jacobi();
        else
            integrate_gs();
        if (p.collision == 1) {
            if (brute_force_collision) self_collision_all_pairs(1); else self_collision_grid(1);
        } else if (p.collision == 2) {
            if (brute_force_collision) self_collision_all_pairs(2); else self_collision_grid(2);
        }
        post_velocity();
    }

    // Extension: max over constraints of |‖xi−xj‖ − rest| / rest.
    T strain_residual() const {
        T r = 0;
        for (size_t e = 0; e < ci.size(); ++e) {
            T len = length(sim_pos[ci[e]] - sim_pos[cj[e]]);
            T s = std::fabs(len - rest[e]) / rest[e];
            if (s > r) r = s;
        }
        return r;
    }
};

// ============================================================================================================
// Extension: spatial-hash collision specification (cell keys, stable LSD radix sort, pair list).
// ============================================================================================================
inline uint32_t hash_cell_key(float x, float y, float z, float inv_cell, uint32_t table_bits) {
    int32_t ix = (int32_t)std::floor(x * inv_cell);
    int32_t iy = (int32_t)std::floor(y * inv_cell);
    int32_t iz = (int32_t)std::floor(z * inv_cell);
    uint32_t h = ((uint32_t)ix * 73856093u) ^ ((uint32_t)iy * 19349663u) ^ ((uint32_t)iz * 83492791u);
    return h & ((1u << table_bits) - 1u);
}
// Stable LSD radix sort, 8-bit digits, `passes` passes from the least significant digit.
inline void stable_radix_sort(std::vector<uint32_t>& keys, std::vector<uint32_t>& vals, int passes) {
    size_t n = keys.size();
    std::vector<uint32_t> k2(n), v2(n);
    for (int pass = 0; pass < passes; ++pass) {
        uint32_t shift = 8u * (uint32_t)pass;
        size_t count[257] = {0};
        for (size_t i = 0; i < n; ++i) count[((keys[i] >> shift) & 0xFF) + 1]++;
        for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
        for (size_t i = 0; i < n; ++i) {
            uint32_t d = (keys[i] >> shift) & 0xFF;
            size_t dst = count[d]++;
            k2[dst] = keys[i];
            v2[dst] = vals[i];
        }
        keys.swap(k2);
        vals.swap(v2);
    }
}

}  // namespace oracle
