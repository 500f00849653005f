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

}  // namespace xpbd
