// CPU check of the spatial-patch tables built for the shared-memory Jacobi kernel: every local index is in range,
// each unpinned particle is owned by exactly one patch, and each owned particle's gather slots reproduce its row of
// the reference neighbour table (mesh_prep.rs:588-635) in order, with the right endpoint sign.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "mesh_prep.h"
#include "xpbd_internal.h"

using namespace xpbd;

static int check(const char* name, uint32_t n, std::vector<float> rest, std::vector<float> w, std::vector<uint32_t> ci,
                 std::vector<uint32_t> cj, uint32_t target, bool expect_ok) {
    const uint32_t e = (uint32_t)ci.size();
    std::vector<uint32_t> perm, colors, offs;
    color_constraints(n, e, ci.data(), cj.data(), false, perm, colors, offs);
    std::vector<uint32_t> si(e), sj(e), spal(e, 0);
    std::vector<float> srest(e, 1.0f);
    for (uint32_t k = 0; k < e; ++k) {
        si[k] = ci[perm[k]];
        sj[k] = cj[perm[k]];
        spal[k] = perm[k] % 3;
    }
    std::vector<uint32_t> roff, other, eid, slot;
    neighbor_csr(n, e, si.data(), sj.data(), roff, other, eid);
    PatchArrays pa;
    const uint32_t base = 1000;  // vertex offset of this cloth in a batch
    bool ok = build_cloth_patches(n, rest.data(), w.data(), e, si.data(), sj.data(), srest.data(), spal.data(), roff,
                                  other, eid, base, 7, target, 4096, pa, slot);
    if (ok != expect_ok) {
        printf("%s: build returned %d, expected %d\n", name, ok, expect_ok);
        return 1;
    }
    if (!ok) {
        printf("%s: ok (rejected as expected)\n", name);
        return 0;
    }
    std::vector<int> owner(n, -1);
    const size_t np_ = pa.header.size() / 6;
    for (size_t p = 0; p < np_; ++p) {
        const uint32_t* h = &pa.header[6 * p];
        const uint32_t parts_off = h[0], con_off = h[1], gofs_off = h[2], npo = h[3] & 0xFFFF, nh = h[3] >> 16,
                       nc = h[4];
        if (h[5] != 7) return printf("%s: cloth id\n", name), 1;
        if (npo + nh > XPBD_PATCH_MAX_LOCAL || nc > XPBD_PATCH_MAX_CON || npo + nh + nc > 4096)
            return printf("%s: patch %zu too big\n", name, p), 1;
        if (npo + nh > pa.max_local || nc > pa.max_con) return printf("%s: max\n", name), 1;
        for (uint32_t k = 0; k < npo; ++k) {
            const uint32_t g = pa.parts[parts_off + k] - base;
            if (g >= n || owner[g] >= 0) return printf("%s: owner\n", name), 1;
            owner[g] = (int)p;
        }
        for (uint32_t c = 0; c < nc; ++c) {
            const uint32_t rx = pa.con[2 * (con_off + c)];
            const uint32_t li = rx & 0xFFF, lj = (rx >> 12) & 0xFFF;
            if (li >= npo + nh || lj >= npo + nh) return printf("%s: local index\n", name), 1;
        }
        for (uint32_t k = 0; k < npo; ++k) {
            const uint32_t g = pa.parts[parts_off + k] - base;
            const uint32_t q0 = pa.gofs[gofs_off + k], q1 = pa.gofs[gofs_off + k + 1];
            if (w[g] <= 0.f) {
                if (q1 != q0) return printf("%s: pinned row not empty\n", name), 1;
                continue;
            }
            if (q1 - q0 != roff[g + 1] - roff[g]) return printf("%s: row length %u\n", name, g), 1;
            for (uint32_t q = q0; q < q1; ++q) {
                const uint32_t sl = pa.slots[q], c = sl & 0x7FFF;
                if (c >= nc) return printf("%s: slot range\n", name), 1;
                const uint32_t rx = pa.con[2 * (con_off + c)];
                const uint32_t li = rx & 0xFFF, lj = (rx >> 12) & 0xFFF;
                const uint32_t self = (sl & 0x8000) ? lj : li, oth = (sl & 0x8000) ? li : lj;
                const uint32_t gself = pa.parts[parts_off + self] - base, goth = pa.parts[parts_off + oth] - base;
                const uint32_t ref = roff[g] + (q - q0);
                if (self != k || gself != g || goth != other[ref]) return printf("%s: row order %u\n", name, g), 1;
                const uint32_t e_ref = eid[ref];
                if (si[e_ref] + 0 != (sl & 0x8000 ? goth : gself) || sj[e_ref] != (sl & 0x8000 ? gself : goth))
                    return printf("%s: endpoint sign\n", name), 1;
                if ((rx >> 24) != spal[e_ref]) return printf("%s: palette\n", name), 1;
            }
        }
    }
    for (uint32_t g = 0; g < n; ++g)
        if (owner[g] < 0) return printf("%s: particle %u unowned\n", name, g), 1;
    printf("%s: ok (%zu patches, max local %u, max constraints %u)\n", name, np_, pa.max_local, pa.max_con);
    return 0;
}

int main() {
    int fails = 0;
    for (uint32_t s : {3u, 17u, 64u, 150u}) {
        const uint32_t n = s * s;
        std::vector<float> rest(3 * n), w(n, 100.f);
        std::vector<uint32_t> ci, cj;
        for (uint32_t r = 0; r < s; ++r)
            for (uint32_t c = 0; c < s; ++c) {
                const uint32_t i = r * s + c;
                rest[3 * i] = (float)c;
                rest[3 * i + 1] = 1.f;
                rest[3 * i + 2] = (float)r;
                if (c + 1 < s) ci.push_back(i), cj.push_back(i + 1);
                if (r + 1 < s) ci.push_back(i), cj.push_back(i + s);
                if (c + 1 < s && r + 1 < s) {
                    ci.push_back(i), cj.push_back(i + s + 1);
                    ci.push_back(i + 1), cj.push_back(i + s);
                }
                if (c + 2 < s) ci.push_back(i), cj.push_back(i + 2);
                if (r + 2 < s) ci.push_back(i), cj.push_back(i + 2 * s);
            }
        for (uint32_t c = 0; c < s; ++c) w[c] = 0.f;  // top edge pinned
        char name[64];
        snprintf(name, sizeof(name), "sheet%u", s);
        fails += check(name, n, rest, w, ci, cj, 256, true);
    }
    {  // random geometric multigraph with duplicate constraints
        std::mt19937 rng(3);
        const uint32_t n = 3000;
        std::vector<float> rest(3 * n), w(n, 1.f);
        for (auto& v : rest) v = (float)(rng() % 1000) / 100.f;
        std::vector<uint32_t> ci, cj;
        for (int k = 0; k < 12000; ++k) {
            uint32_t a = rng() % n, b = rng() % n;
            if (a != b) ci.push_back(a), cj.push_back(b);
        }
        for (uint32_t k = 0; k < n; k += 17) w[k] = 0.f;
        fails += check("random", n, rest, w, ci, cj, 200, true);
    }
    {  // a particle with more constraints than a patch can hold
        const uint32_t n = 6000;
        std::vector<float> rest(3 * n, 0.f), w(n, 1.f);
        std::vector<uint32_t> ci, cj;
        for (uint32_t k = 1; k < n; ++k) ci.push_back(0), cj.push_back(k);
        fails += check("star", n, rest, w, ci, cj, 256, false);
    }
    return fails ? 1 : 0;
}
