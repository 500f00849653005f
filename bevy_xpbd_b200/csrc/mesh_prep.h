// Host-side topology preparation (mesh_prep.cpp).
#pragma once
#include <stdint.h>

#include <vector>

namespace xpbd {

// Greedy edge coloring in the reference processing order (index_order=false) or plain index order. perm[k] is the
// input index of the k-th batch-sorted constraint, colors_sorted its color, offsets the batch starts + total.
void color_constraints(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, bool index_order,
                       std::vector<uint32_t>& perm, std::vector<uint32_t>& colors_sorted,
                       std::vector<uint32_t>& offsets);

// Particle-major incidence table from batch-sorted constraints (cursor-scatter order).
void neighbor_csr(uint32_t n, uint32_t e_count, const uint32_t* ci_sorted, const uint32_t* cj_sorted,
                  std::vector<uint32_t>& row_off, std::vector<uint32_t>& other, std::vector<uint32_t>& eid);

// Appends the sorted `depth`-ring of each particle (indices offset by `base`) to idx/off; `off` gets n entries
// appended after its current last value (pass off = {} for a fresh table: a leading 0 is inserted).
void topology_rings(uint32_t n, uint32_t e_count, const uint32_t* ci, const uint32_t* cj, const uint32_t* ctype,
                    uint32_t depth, uint32_t base, std::vector<uint32_t>& off, std::vector<uint32_t>& idx);

// Spatial patches of one cloth for the shared-memory Jacobi kernel (see XpbdPatch). Particles are split by recursive
// coordinate bisection of their rest positions into blocks of at most `target` particles (further while a patch's
// particles + halo exceed XPBD_PATCH_MAX_LOCAL, its constraints XPBD_PATCH_MAX_CON, or both `max_entries`). Inputs are
// the cloth's batch-sorted constraints (si, sj, rest, palette index) and their neighbour table (row_off, other, eid).
// Appends to the batch arrays; slot_of_con[e] receives the global slot of sorted constraint e (first patch holding
// it, UINT32_MAX if none). Returns false if a single particle cannot fit a patch.
struct PatchArrays {
    std::vector<uint32_t> header;  // 6 u32 per patch: parts_off, con_off, gofs_off, np | nh << 16, nc, cloth
    std::vector<uint32_t> parts;
    std::vector<uint32_t> con;     // 2 u32 per record
    std::vector<uint32_t> gofs;
    std::vector<uint16_t> slots;
    uint32_t max_local = 0, max_con = 0;
};
bool build_cloth_patches(uint32_t n, const float* rest_xyz, const float* inv_mass, uint32_t e_count,
                         const uint32_t* si, const uint32_t* sj, const float* srest, const uint32_t* spal,
                         const std::vector<uint32_t>& row_off, const std::vector<uint32_t>& other,
                         const std::vector<uint32_t>& eid, uint32_t vtx_off, uint32_t cloth, uint32_t target,
                         uint32_t max_entries, PatchArrays& out, std::vector<uint32_t>& slot_of_con);

}  // namespace xpbd
