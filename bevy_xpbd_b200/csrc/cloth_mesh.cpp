// Cloth mesh builders: the host-side mesh preparation of the reference crate (src/mesh_prep.rs) that turns a
// triangle mesh into the solver's inputs — inverse masses from triangle areas, top-row pins, structural edge
// constraints, hinge bending constraints, extra braces, greedy-colored batch order.
//
//   xpbd_mesh_grid_hanging  grid_cloth_hanging        (mesh_prep.rs:363-406, cross diagonals :409-426, braces :504-530)
//   xpbd_mesh_from_obj      parse_welded_obj          (mesh_prep.rs:223-357, grid braces :444-501)
//   xpbd_mesh_from_triangles finalize_cloth_mesh      (mesh_prep.rs:532-659) with caller-given extra constraints
//
// Floating-point steps follow the reference's f32 operations in order (glam: length = sqrt((x·x + y·y) + z·z),
// cross = (y·z' − z·y', z·x' − x·z', x·y' − y·x')); strtof parses like Rust's str::parse::<f32> (correctly rounded).
// Dedup sets keep the first occurrence in iteration order, which is what the reference's HashMap-insert tests give.
#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/xpbd_cuda.h"
#include "mesh_prep.h"

namespace {

constexpr float kStretchComp = 2e-8f;   // DEFAULT_STRETCH_COMPLIANCE, mesh_prep.rs:93
constexpr float kBendComp = 3.8f;       // DEFAULT_BEND_COMPLIANCE, mesh_prep.rs:89
constexpr float kSkip2Comp = 2.5e-8f;   // DEFAULT_SKIP2_COMPLIANCE, mesh_prep.rs:97
constexpr float kCrossComp = 6e-9f;     // DEFAULT_CROSS_DIAG_COMPLIANCE, mesh_prep.rs:101

struct P3 {
    float x, y, z;
};
inline P3 minus(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float length(P3 a) { return sqrtf((a.x * a.x + a.y * a.y) + a.z * a.z); }
inline float distance(P3 a, P3 b) { return length(minus(a, b)); }
inline P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

struct Link {
    uint32_t i, j;
    float rest, comp;
};

inline uint64_t pair_key(uint32_t a, uint32_t b) { return ((uint64_t)a << 32) | b; }

}  // namespace

struct xpbd_mesh {
    std::vector<P3> pos;
    std::vector<uint32_t> tris;
    std::vector<float> inv_mass;
    std::vector<Link> links;          // batch-sorted
    std::vector<uint32_t> batch_off;  // batch starts + total
};

namespace {

// For each triangle edge slot 3t + k (edge from corner k to corner k+1), the slot of the same edge in another
// triangle, or UINT32_MAX. Edges are ordered by (min, max) keeping slot order among equals, and every adjacent equal
// pair is linked in that order (so a slot shared three ways keeps its last partner), as find_tri_neighbors does
// (mesh_prep.rs:660-693).
std::vector<uint32_t> edge_partners(const std::vector<uint32_t>& tris) {
    const uint32_t slots = (uint32_t)tris.size();
    std::vector<uint64_t> key(slots);
    std::vector<uint32_t> order(slots);
    for (uint32_t s = 0; s < slots; ++s) {
        const uint32_t t = s / 3, k = s % 3;
        const uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
        key[s] = pair_key(std::min(a, b), std::max(a, b));
        order[s] = s;
    }
    std::stable_sort(order.begin(), order.end(), [&](uint32_t p, uint32_t q) { return key[p] < key[q]; });
    std::vector<uint32_t> partner(slots, 0xFFFFFFFFu);
    for (uint32_t r = 0; r + 1 < slots; ++r) {
        const uint32_t p = order[r], q = order[r + 1];
        if (key[p] == key[q]) {
            partner[p] = q;
            partner[q] = p;
        }
    }
    return partner;
}

xpbd_mesh* finalize(std::vector<P3> pos, std::vector<uint32_t> tris, const std::vector<Link>& extras) {
    auto* m = new xpbd_mesh();
    const uint32_t n = (uint32_t)pos.size();
    const uint32_t nt = (uint32_t)(tris.size() / 3);
    tris.resize(3 * (size_t)nt);
    // inverse mass: a third of 1/area of every incident triangle (unit density), mesh_prep.rs:539-552
    m->inv_mass.assign(n, 0.0f);
    for (uint32_t t = 0; t < nt; ++t) {
        const uint32_t a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
        const float area = 0.5f * length(cross(minus(pos[b], pos[a]), minus(pos[c], pos[a])));
        const float share = area > 0.0f ? 1.0f / area / 3.0f : 0.0f;
        m->inv_mass[a] += share;
        m->inv_mass[b] += share;
        m->inv_mass[c] += share;
    }
    const std::vector<uint32_t> partner = edge_partners(tris);
    // the top row (y within 1e-5 of the maximum) is pinned, mesh_prep.rs:556-566
    float top = -INFINITY;
    for (const P3& p : pos) top = fmaxf(top, p.y);
    for (uint32_t v = 0; v < n; ++v)
        if (pos[v].y >= top - 1e-5f) m->inv_mass[v] = 0.0f;
    std::vector<Link> links;
    // structural edges: an interior edge once (from the slot whose first corner has the smaller index), a boundary
    // edge from its slot; first occurrence wins, mesh_prep.rs:695-719
    {
        std::unordered_map<uint64_t, char> seen;
        seen.reserve(2 * tris.size());
        for (uint32_t s = 0; s < 3 * nt; ++s) {
            const uint32_t t = s / 3, k = s % 3;
            const uint32_t a = tris[3 * t + k], b = tris[3 * t + (k + 1) % 3];
            if (partner[s] != 0xFFFFFFFFu && a >= b) continue;
            const uint32_t lo = std::min(a, b), hi = std::max(a, b);
            if (!seen.emplace(pair_key(lo, hi), 1).second) continue;
            links.push_back({lo, hi, distance(pos[lo], pos[hi]), kStretchComp});
        }
    }
    // hinge bending: the two corners opposite a shared edge, mesh_prep.rs:721-744
    {
        std::unordered_map<uint64_t, char> seen;
        seen.reserve(2 * tris.size());
        for (uint32_t s = 0; s < 3 * nt; ++s) {
            const uint32_t q = partner[s];
            if (q == 0xFFFFFFFFu) continue;
            const uint32_t t = s / 3, k = s % 3;
            const uint32_t c0 = tris[3 * t + (k + 2) % 3];
            const uint32_t c1 = tris[3 * (q / 3) + (q % 3 + 2) % 3];
            const uint32_t lo = std::min(c0, c1), hi = std::max(c0, c1);
            if (!seen.emplace(pair_key(lo, hi), 1).second) continue;
            links.push_back({lo, hi, distance(pos[lo], pos[hi]), kBendComp});
        }
    }
    links.insert(links.end(), extras.begin(), extras.end());
    // greedy-colored batches in the reference's processing order
    std::vector<uint32_t> ci(links.size()), cj(links.size()), perm, colors;
    for (size_t e = 0; e < links.size(); ++e) {
        ci[e] = links[e].i;
        cj[e] = links[e].j;
    }
    xpbd::color_constraints(n, (uint32_t)links.size(), ci.data(), cj.data(), false, perm, colors, m->batch_off);
    m->links.resize(links.size());
    for (size_t k = 0; k < links.size(); ++k) m->links[k] = links[perm[k]];
    m->pos = std::move(pos);
    m->tris = std::move(tris);
    return m;
}

// Every-other-vertex braces along the rows, then along the columns, of a cols × rows vertex grid whose vertex at
// (ix, iy) is at(ix, iy); each pair (min, max) with rest = |p_i − p_j|.
template <typename At>
void skip_two_braces(uint32_t cols, uint32_t rows, At at, const std::vector<P3>& pos, std::vector<Link>& out) {
    for (uint32_t iy = 0; iy < rows; ++iy)
        for (uint32_t ix = 0; ix + 2 < cols; ++ix) {
            const uint32_t i = at(ix, iy), j = at(ix + 2, iy);
            out.push_back({std::min(i, j), std::max(i, j), distance(pos[i], pos[j]), kSkip2Comp});
        }
    for (uint32_t iy = 0; iy + 2 < rows; ++iy)
        for (uint32_t ix = 0; ix < cols; ++ix) {
            const uint32_t i = at(ix, iy), j = at(ix, iy + 2);
            out.push_back({std::min(i, j), std::max(i, j), distance(pos[i], pos[j]), kSkip2Comp});
        }
}

// Distinct values within 2e-4 after sorting (each kept value is the first of its run), mesh_prep.rs:429-440.
std::vector<float> grid_lines(std::vector<float> v) {
    std::sort(v.begin(), v.end());
    std::vector<float> out;
    for (float x : v)
        if (out.empty() || fabsf(x - out.back()) > 2e-4f) out.push_back(x);
    return out;
}

// When the vertices are exactly the nodes of a Cartesian grid in x/y, the braces of a subdivided sheet
// (mesh_prep.rs:444-501); otherwise none.
bool grid_braces_if_regular(const std::vector<P3>& pos, std::vector<Link>& out) {
    if (pos.empty()) return false;
    std::vector<float> xs, ys;
    for (const P3& p : pos) {
        xs.push_back(p.x);
        ys.push_back(p.y);
    }
    xs = grid_lines(std::move(xs));
    ys = grid_lines(std::move(ys));
    const size_t cols = xs.size(), rows = ys.size();
    if (cols < 3 || rows < 3 || cols * rows != pos.size()) return false;
    std::vector<uint32_t> at(cols * rows, 0xFFFFFFFFu);
    for (uint32_t v = 0; v < pos.size(); ++v) {
        size_t ix = 0, iy = 0;
        while (ix < cols && !(fabsf(xs[ix] - pos[v].x) <= 2e-4f)) ++ix;  // first grid line within tolerance
        while (iy < rows && !(fabsf(ys[iy] - pos[v].y) <= 2e-4f)) ++iy;
        if (ix == cols || iy == rows) return false;
        uint32_t& slot = at[iy * cols + ix];
        if (slot != 0xFFFFFFFFu) return false;
        slot = v;
    }
    skip_two_braces((uint32_t)cols, (uint32_t)rows, [&](uint32_t ix, uint32_t iy) { return at[iy * cols + ix]; },
                    pos, out);
    return true;
}

}  // namespace

extern "C" int xpbd_mesh_grid_hanging(uint32_t quad_cols, uint32_t quad_rows, float cell_size, xpbd_mesh** out) {
    if (!out || quad_cols < 1 || quad_rows < 1 || !(cell_size > 0.0f) || !isfinite(cell_size))
        return XPBD_ERR_INVALID_ARGUMENT;
    const uint32_t vc = quad_cols + 1, vr = quad_rows + 1;
    std::vector<P3> pos;
    pos.reserve((size_t)vc * vr);
    const float x0 = -0.5f * ((float)quad_cols * cell_size);
    for (uint32_t iy = 0; iy < vr; ++iy)
        for (uint32_t ix = 0; ix < vc; ++ix) pos.push_back({x0 + (float)ix * cell_size, (float)iy * cell_size, 0.0f});
    std::vector<uint32_t> tris;
    tris.reserve(6 * (size_t)quad_cols * quad_rows);
    for (uint32_t iy = 0; iy < quad_rows; ++iy)
        for (uint32_t ix = 0; ix < quad_cols; ++ix) {
            const uint32_t a = iy * vc + ix, b = a + 1, c = a + vc, d = c + 1;
            const uint32_t quad[6] = {a, b, c, b, d, c};
            tris.insert(tris.end(), quad, quad + 6);
        }
    std::vector<Link> extras;
    skip_two_braces(vc, vr, [&](uint32_t ix, uint32_t iy) { return iy * vc + ix; }, pos, extras);
    for (uint32_t iy = 0; iy < quad_rows; ++iy)  // the diagonal the triangle split does not have
        for (uint32_t ix = 0; ix < quad_cols; ++ix) {
            const uint32_t a = iy * vc + ix, d = (iy + 1) * vc + ix + 1;
            extras.push_back({std::min(a, d), std::max(a, d), distance(pos[a], pos[d]), kCrossComp});
        }
    *out = finalize(std::move(pos), std::move(tris), extras);
    return XPBD_OK;
}

extern "C" int xpbd_mesh_from_obj(const char* text, xpbd_mesh** out) {
    if (!text || !out) return XPBD_ERR_INVALID_ARGUMENT;
    std::vector<P3> vpos;
    std::vector<std::vector<std::string>> faces;
    const char* p = text;
    while (*p) {
        const char* e = strchr(p, '\n');
        std::string line(p, e ? (size_t)(e - p) : strlen(p));
        p = e ? e + 1 : p + line.size();
        std::vector<std::string> tok;
        size_t k = 0;
        while (k < line.size()) {  // whitespace-separated tokens
            while (k < line.size() && isspace((unsigned char)line[k])) ++k;
            size_t s = k;
            while (k < line.size() && !isspace((unsigned char)line[k])) ++k;
            if (k > s) tok.emplace_back(line.substr(s, k - s));
        }
        if (tok.empty() || tok[0][0] == '#') continue;
        if (tok[0] == "v") {
            float c[3] = {0.0f, 0.0f, 0.0f};
            for (int q = 0; q < 3 && q + 1 < (int)tok.size(); ++q) {
                char* end = nullptr;
                const float f = strtof(tok[q + 1].c_str(), &end);
                if (end && *end == '\0' && end != tok[q + 1].c_str()) c[q] = f;
            }
            vpos.push_back({c[0], c[1], c[2]});
        } else if (tok[0] == "f") {
            faces.emplace_back(tok.begin() + 1, tok.end());
        }
    }
    // welded corners: one vertex per distinct corner string "v/vt/vn", in order of first use
    std::unordered_map<std::string, uint32_t> corner;
    std::vector<P3> pos;
    auto vertex_of = [&](const std::string& s) {
        auto it = corner.find(s);
        if (it != corner.end()) return it->second;
        const uint32_t id = (uint32_t)pos.size();
        corner.emplace(s, id);
        const std::string first = s.substr(0, s.find('/'));
        size_t vi = 0;  // 1-based in the file; a missing or unparsable index counts as 1; index 0 stays 0
        {
            const bool digits = !first.empty() && first.find_first_not_of("0123456789", first[0] == '+' ? 1 : 0) ==
                                                      std::string::npos && first != "+";
            errno = 0;
            const unsigned long long v = digits ? strtoull(first.c_str(), nullptr, 10) : 1ull;
            vi = (digits && errno == 0) ? (v > 0 ? (size_t)v - 1 : 0) : 0;
        }
        pos.push_back(vi < vpos.size() ? vpos[vi] : P3{0.0f, 0.0f, 0.0f});
        return id;
    };
    std::vector<uint32_t> tris;
    std::vector<Link> cross_links;
    for (const auto& f : faces) {
        if (f.size() < 3) continue;
        if (f.size() == 4) {  // quad split v0-v2 (a triangle fan), the other diagonal v1-v3 as a brace
            const uint32_t v0 = vertex_of(f[0]), v1 = vertex_of(f[1]), v2 = vertex_of(f[2]), v3 = vertex_of(f[3]);
            const uint32_t quad[6] = {v0, v1, v2, v0, v2, v3};
            tris.insert(tris.end(), quad, quad + 6);
            cross_links.push_back({std::min(v1, v3), std::max(v1, v3), 0.0f, kCrossComp});
            continue;
        }
        const uint32_t c0 = vertex_of(f[0]);
        for (size_t q = 1; q + 1 < f.size(); ++q) {
            const uint32_t c1 = vertex_of(f[q]);
            const uint32_t c2 = vertex_of(f[q + 1]);
            tris.push_back(c0);
            tris.push_back(c1);
            tris.push_back(c2);
        }
    }
    for (Link& l : cross_links) l.rest = distance(pos[l.i], pos[l.j]);
    std::vector<Link> extras;
    grid_braces_if_regular(pos, extras);
    extras.insert(extras.end(), cross_links.begin(), cross_links.end());
    *out = finalize(std::move(pos), std::move(tris), extras);
    return XPBD_OK;
}

extern "C" int xpbd_mesh_from_triangles(uint32_t num_vertices, const float* positions, uint32_t num_tris,
                                        const uint32_t* tri_indices, uint32_t num_extra, const uint32_t* extra_i,
                                        const uint32_t* extra_j, const float* extra_rest, const float* extra_comp,
                                        xpbd_mesh** out) {
    if (!out || (num_vertices && !positions) || (num_tris && !tri_indices) ||
        (num_extra && (!extra_i || !extra_j || !extra_rest || !extra_comp)))
        return XPBD_ERR_INVALID_ARGUMENT;
    for (size_t k = 0; k < 3 * (size_t)num_tris; ++k)
        if (tri_indices[k] >= num_vertices) return XPBD_ERR_INDEX_RANGE;
    std::vector<P3> pos(num_vertices);
    for (uint32_t v = 0; v < num_vertices; ++v) pos[v] = {positions[3 * v], positions[3 * v + 1], positions[3 * v + 2]};
    std::vector<Link> extras(num_extra);
    for (uint32_t k = 0; k < num_extra; ++k) {
        if (extra_i[k] >= num_vertices || extra_j[k] >= num_vertices || extra_i[k] == extra_j[k])
            return XPBD_ERR_INDEX_RANGE;
        extras[k] = {extra_i[k], extra_j[k], extra_rest[k], extra_comp[k]};
    }
    *out = finalize(std::move(pos), std::vector<uint32_t>(tri_indices, tri_indices + 3 * (size_t)num_tris), extras);
    return XPBD_OK;
}

extern "C" int xpbd_mesh_sizes(const xpbd_mesh* m, uint32_t* num_vertices, uint32_t* num_tris,
                               uint32_t* num_constraints, uint32_t* num_batches) {
    if (!m) return XPBD_ERR_INVALID_ARGUMENT;
    if (num_vertices) *num_vertices = (uint32_t)m->pos.size();
    if (num_tris) *num_tris = (uint32_t)(m->tris.size() / 3);
    if (num_constraints) *num_constraints = (uint32_t)m->links.size();
    if (num_batches) *num_batches = (uint32_t)m->batch_off.size() - 1;
    return XPBD_OK;
}

extern "C" int xpbd_mesh_get(const xpbd_mesh* m, float* positions, float* inv_mass, uint32_t* tri_indices,
                             uint32_t* constraint_i, uint32_t* constraint_j, float* rest_len, float* compliance,
                             uint32_t* batch_offsets) {
    if (!m) return XPBD_ERR_INVALID_ARGUMENT;
    for (size_t v = 0; v < m->pos.size(); ++v) {
        if (positions) {
            positions[3 * v] = m->pos[v].x;
            positions[3 * v + 1] = m->pos[v].y;
            positions[3 * v + 2] = m->pos[v].z;
        }
        if (inv_mass) inv_mass[v] = m->inv_mass[v];
    }
    if (tri_indices) std::copy(m->tris.begin(), m->tris.end(), tri_indices);
    for (size_t e = 0; e < m->links.size(); ++e) {
        if (constraint_i) constraint_i[e] = m->links[e].i;
        if (constraint_j) constraint_j[e] = m->links[e].j;
        if (rest_len) rest_len[e] = m->links[e].rest;
        if (compliance) compliance[e] = m->links[e].comp;
    }
    if (batch_offsets) std::copy(m->batch_off.begin(), m->batch_off.end(), batch_offsets);
    return XPBD_OK;
}

extern "C" void xpbd_mesh_free(xpbd_mesh* m) { delete m; }
