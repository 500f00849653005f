// Host-side topology preparation for the packed batch (runs once per xpbd_commit).
//
//   color_constraints      greedy edge coloring with the processing order of partition_constraints_for_gs_batches
//                          (mesh_prep.rs:153-221): edges ordered by (max endpoint degree descending, min endpoint,
//                          max endpoint, index); each takes the smallest color free at both endpoints; batches are
//                          (color, index) ordered. Implemented with a degree-bucketed ordering and per-particle
//                          64-bit color masks (O(E log E)), producing the same coloring as the reference.
//   neighbor_csr           particle-major incidence table in the cursor-scatter order of finalize_cloth_mesh
//                          (mesh_prep.rs:588-635): row i lists i's constraints in batch-sorted constraint order.
//   topology_rings         sorted k-ring neighbourhoods over stretch/shear edges (collision ring filter).
#include "mesh_prep.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "xpbd_internal.h"

namespace xpbd {

void color_constraints(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, bool index_order,
                       std::vector<uint32_t>& perm, std::vector<uint32_t>& colors_sorted,
                       std::vector<uint32_t>& offsets) {
    perm.assign(e_count, 0);
    colors_sorted.assign(e_count, 0);
    offsets.clear();
    if (e_count == 0) {
        offsets = {0, 0};
        return;
    }
    std::vector<uint32_t> deg(n, 0);
    for (uint32_t e = 0; e < e_count; ++e) {
        ++deg[ci[e]];
        ++deg[cj[e]];
    }
    // processing order
    std::vector<uint32_t> order(e_count);
    if (index_order) {
        for (uint32_t e = 0; e < e_count; ++e) order[e] = e;
    } else {
        uint32_t maxd = 0;
        std::vector<uint32_t> dkey(e_count);
        for (uint32_t e = 0; e < e_count; ++e) {
            dkey[e] = std::max(deg[ci[e]], deg[cj[e]]);
            maxd = std::max(maxd, dkey[e]);
        }
        // bucket by degree, highest first
        std::vector<uint32_t> start(maxd + 2, 0);
        for (uint32_t e = 0; e < e_count; ++e) ++start[maxd - dkey[e] + 1];
        for (uint32_t d = 0; d <= maxd; ++d) start[d + 1] += start[d];
        std::vector<uint32_t> bucketed(e_count);
        {
            std::vector<uint32_t> cur(start.begin(), start.end() - 1);
            for (uint32_t e = 0; e < e_count; ++e) bucketed[cur[maxd - dkey[e]]++] = e;
        }
        // within a bucket: (min endpoint, max endpoint, index) ascending
        struct K {
            uint64_t mm;
            uint32_t e;
        };
        std::vector<K> tmp;
        for (uint32_t d = 0; d <= maxd; ++d) {
            uint32_t a = start[d], b = start[d + 1];
            tmp.resize(b - a);
            for (uint32_t k = a; k < b; ++k) {
                uint32_t e = bucketed[k];
                uint64_t lo = std::min(ci[e], cj[e]), hi = std::max(ci[e], cj[e]);
                tmp[k - a] = {(lo << 32) | hi, e};
            }
            std::sort(tmp.begin(), tmp.end(), [](const K& x, const K& y) {
                return x.mm != y.mm ? x.mm < y.mm : x.e < y.e;
            });
            for (uint32_t k = a; k < b; ++k) order[k] = tmp[k - a].e;
        }
    }
    // greedy: smallest color unused at both endpoints
    std::vector<uint64_t> used(n, 0);
    std::vector<std::vector<uint32_t>> used_hi;  // colors >= 64, rarely needed
    std::vector<uint32_t> color(e_count, 0);
    uint32_t ncolors = 0;
    for (uint32_t e : order) {
        const uint32_t i = ci[e], j = cj[e];
        const uint64_t m = used[i] | used[j];
        uint32_t c;
        if (m != ~0ull) {
            c = (uint32_t)__builtin_ctzll(~m);
        } else {
            if (used_hi.empty()) used_hi.resize(n);
            c = 64;
            auto taken = [&](uint32_t col) {
                return std::find(used_hi[i].begin(), used_hi[i].end(), col) != used_hi[i].end() ||
                       std::find(used_hi[j].begin(), used_hi[j].end(), col) != used_hi[j].end();
            };
            while (taken(c)) ++c;
        }
        color[e] = c;
        if (c < 64) {
            used[i] |= 1ull << c;
            used[j] |= 1ull << c;
        } else {
            used_hi[i].push_back(c);
            used_hi[j].push_back(c);
        }
        ncolors = std::max(ncolors, c + 1);
    }
    // (color, index) order by a stable counting sort on color
    std::vector<uint32_t> cstart(ncolors + 1, 0);
    for (uint32_t e = 0; e < e_count; ++e) ++cstart[color[e] + 1];
    for (uint32_t c = 0; c < ncolors; ++c) cstart[c + 1] += cstart[c];
    std::vector<uint32_t> cur(cstart.begin(), cstart.end() - 1);
    for (uint32_t e = 0; e < e_count; ++e) {
        uint32_t p = cur[color[e]]++;
        perm[p] = e;
        colors_sorted[p] = color[e];
    }
    // batch offsets at color changes (colors may be skipped only if unused, which greedy never does)
    offsets.push_back(0);
    for (uint32_t c = 0; c < ncolors; ++c)
        if (cstart[c + 1] > cstart[c] && cstart[c] > 0) offsets.push_back(cstart[c]);
    offsets.push_back(e_count);
}

void neighbor_csr(uint32_t n, uint32_t e_count, const uint32_t* ci_sorted, const uint32_t* cj_sorted,
                  std::vector<uint32_t>& row_off, std::vector<uint32_t>& other, std::vector<uint32_t>& eid) {
    row_off.assign(n + 1, 0);
    for (uint32_t e = 0; e < e_count; ++e) {
        ++row_off[ci_sorted[e] + 1];
        ++row_off[cj_sorted[e] + 1];
    }
    for (uint32_t i = 0; i < n; ++i) row_off[i + 1] += row_off[i];
    other.resize(row_off[n]);
    eid.resize(row_off[n]);
    std::vector<uint32_t> cur(row_off.begin(), row_off.end() - 1);
    for (uint32_t e = 0; e < e_count; ++e) {
        const uint32_t i = ci_sorted[e], j = cj_sorted[e];
        uint32_t p = cur[i]++;
        other[p] = j;
        eid[p] = e;
        p = cur[j]++;
        other[p] = i;
        eid[p] = e;
    }
}

void topology_rings(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, const uint32_t* ctype,
                    uint32_t depth, uint32_t base, std::vector<uint32_t>& off, std::vector<uint32_t>& idx) {
    // adjacency over stretch / shear constraints
    std::vector<uint32_t> aoff(n + 1, 0);
    for (uint32_t e = 0; e < e_count; ++e)
        if (!ctype || ctype[e] <= 1) {
            ++aoff[ci[e] + 1];
            ++aoff[cj[e] + 1];
        }
    for (uint32_t i = 0; i < n; ++i) aoff[i + 1] += aoff[i];
    std::vector<uint32_t> adj(aoff[n]);
    {
        std::vector<uint32_t> cur(aoff.begin(), aoff.end() - 1);
        for (uint32_t e = 0; e < e_count; ++e)
            if (!ctype || ctype[e] <= 1) {
                adj[cur[ci[e]]++] = cj[e];
                adj[cur[cj[e]]++] = ci[e];
            }
    }
    const size_t off0 = idx.size();
    if (off.empty()) off.push_back(0);
    std::vector<uint32_t> frontier, next, ring;
    std::vector<uint32_t> mark(n, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < n; ++i) {
        ring.clear();
        frontier.assign(1, i);
        mark[i] = i;
        for (uint32_t d = 0; d < depth; ++d) {
            next.clear();
            for (uint32_t u : frontier)
                for (uint32_t k = aoff[u]; k < aoff[u + 1]; ++k) {
                    uint32_t v = adj[k];
                    if (mark[v] != i) {
                        mark[v] = i;
                        next.push_back(v);
                        ring.push_back(v);
                    }
                }
            frontier.swap(next);
        }
        std::sort(ring.begin(), ring.end());
        for (uint32_t v : ring) idx.push_back(v + base);
        off.push_back((uint32_t)idx.size());
    }
    (void)off0;
}

namespace {
struct PatchBuilder {
    uint32_t n;
    const float* rest;
    const float* w;
    const uint32_t *si, *sj, *spal;
    const float* srest;
    const std::vector<uint32_t>&row_off, &other, &eid;
    uint32_t vtx_off, cloth, target, max_entries;
    PatchArrays& out;
    std::vector<uint32_t>& slot_of_con;
    std::vector<int32_t> local;      // particle -> local index in the current patch, -1 otherwise
    std::vector<int32_t> con_slot;   // sorted constraint -> slot in the current patch, -1 otherwise
    std::vector<uint32_t> ids;

    bool emit(uint32_t lo, uint32_t hi) {
        std::vector<uint32_t> owned(ids.begin() + lo, ids.begin() + hi);
        std::sort(owned.begin(), owned.end());
        for (uint32_t k = 0; k < owned.size(); ++k) local[owned[k]] = (int32_t)k;
        std::vector<uint32_t> halo, cons;
        for (uint32_t p : owned) {
            if (w[p] <= 0.f) continue;  // only unpinned particles gather; their constraints are all a patch needs
            for (uint32_t q = row_off[p]; q < row_off[p + 1]; ++q) {
                const uint32_t e = eid[q];
                if (con_slot[e] < 0) {
                    con_slot[e] = 0;
                    cons.push_back(e);
                }
                const uint32_t o = other[q];
                if (local[o] == -1) {
                    local[o] = -2;  // provisional halo mark
                    halo.push_back(o);
                }
            }
        }
        std::sort(halo.begin(), halo.end());
        std::sort(cons.begin(), cons.end());
        const size_t nl = owned.size() + halo.size();
        bool ok = nl <= XPBD_PATCH_MAX_LOCAL && cons.size() <= XPBD_PATCH_MAX_CON && nl + cons.size() <= max_entries &&
                  owned.size() <= 0xFFFF && halo.size() <= 0xFFFF;
        if (ok) {
            for (uint32_t k = 0; k < halo.size(); ++k) local[halo[k]] = (int32_t)(owned.size() + k);
            for (uint32_t k = 0; k < cons.size(); ++k) con_slot[cons[k]] = (int32_t)k;
            const uint32_t parts_off = (uint32_t)out.parts.size();
            const uint32_t con_off = (uint32_t)(out.con.size() / 2);
            const uint32_t gofs_off = (uint32_t)out.gofs.size();
            for (uint32_t p : owned) out.parts.push_back(p + vtx_off);
            for (uint32_t p : halo) out.parts.push_back(p + vtx_off);
            for (uint32_t e : cons) {
                const uint32_t li = (uint32_t)local[si[e]], lj = (uint32_t)local[sj[e]];
                uint32_t rb;
                memcpy(&rb, &srest[e], 4);
                out.con.push_back(li | (lj << 12) | (spal[e] << 24));
                out.con.push_back(rb);
                if (slot_of_con[e] == 0xFFFFFFFFu) slot_of_con[e] = con_off + (uint32_t)con_slot[e];
            }
            for (uint32_t p : owned) {
                out.gofs.push_back((uint32_t)out.slots.size());
                if (w[p] <= 0.f) continue;  // pinned: jacobi_gather returns jac_in unchanged
                for (uint32_t q = row_off[p]; q < row_off[p + 1]; ++q) {
                    const uint32_t e = eid[q];
                    out.slots.push_back((uint16_t)((uint32_t)con_slot[e] | (sj[e] == p ? 0x8000u : 0u)));
                }
            }
            out.gofs.push_back((uint32_t)out.slots.size());
            out.header.insert(out.header.end(), {parts_off, con_off, gofs_off,
                                                 (uint32_t)owned.size() | ((uint32_t)halo.size() << 16),
                                                 (uint32_t)cons.size(), cloth});
            out.max_local = std::max<uint32_t>(out.max_local, (uint32_t)nl);
            out.max_con = std::max<uint32_t>(out.max_con, (uint32_t)cons.size());
        }
        for (uint32_t p : owned) local[p] = -1;
        for (uint32_t p : halo) local[p] = -1;
        for (uint32_t e : cons) con_slot[e] = -1;
        return ok;
    }

    bool split(uint32_t lo, uint32_t hi, bool force) {
        if (!force && hi - lo <= target) {
            if (emit(lo, hi)) return true;
            if (hi - lo == 1) return false;
        }
        if (hi - lo <= 1) return emit(lo, hi);
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t k = lo; k < hi; ++k)
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::min(mn[a], rest[3 * ids[k] + a]);
                mx[a] = std::max(mx[a], rest[3 * ids[k] + a]);
            }
        int axis = 0;
        for (int a = 1; a < 3; ++a)
            if (mx[a] - mn[a] > mx[axis] - mn[axis]) axis = a;
        const uint32_t mid = lo + (hi - lo) / 2;
        std::nth_element(ids.begin() + lo, ids.begin() + mid, ids.begin() + hi, [&](uint32_t x, uint32_t y) {
            const float cx = rest[3 * x + axis], cy = rest[3 * y + axis];
            return cx != cy ? cx < cy : x < y;
        });
        return split(lo, mid, false) && split(mid, hi, false);
    }
};
}  // namespace

bool build_cloth_patches(uint32_t n, const float* rest_xyz, const float* inv_mass, uint32_t e_count,
                         const uint32_t* si, const uint32_t* sj, const float* srest, const uint32_t* spal,
                         const std::vector<uint32_t>& row_off, const std::vector<uint32_t>& other,
                         const std::vector<uint32_t>& eid, uint32_t vtx_off, uint32_t cloth, uint32_t target,
                         uint32_t max_entries, PatchArrays& out, std::vector<uint32_t>& slot_of_con) {
    slot_of_con.assign(e_count, 0xFFFFFFFFu);
    PatchBuilder b{n, rest_xyz, inv_mass, si, sj, spal, srest, row_off, other, eid, vtx_off, cloth, target,
                   max_entries, out, slot_of_con, std::vector<int32_t>(n, -1), std::vector<int32_t>(e_count, -1),
                   std::vector<uint32_t>(n)};
    for (uint32_t k = 0; k < n; ++k) b.ids[k] = k;
    return b.split(0, n, false);
}

}  // namespace xpbd
