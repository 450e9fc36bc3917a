// pms_pattern.h -- CSR pattern of the global matrix and the deterministic gather maps.
//
// The reference assembles K as COO triplets with duplicates in cell order and lets the
// sparse solver sum them (src/base/assembly.rs:70-139, src/fem/linear_system.rs:132-164).
// Here the pattern is built once per mesh.  Block row A of K (node A, ND x ND blocks) is the sum,
// over the cells incident to A in ascending cell order, of the node-row slab (a, all b) of each
// cell's dense element matrix, where a is A's local index in the cell.  The gather kernel owns
// one block row, adds the slabs in that fixed order and writes the row once; slot[] says where
// each local column node b of an incidence lands in the row.  No atomics: the same bits on every
// run, and the same bits as summing each node-pair block over its cells in ascending order.
#pragma once
#include <cstdint>
#include <vector>

namespace pms {

struct Pattern {
    int nd = 0, nn = 0;
    int64_t npoint = 0, ncell = 0;
    // node -> (cell*nn + local) incidences, ascending cell
    std::vector<int64_t> inc_ptr;
    std::vector<int32_t> inc;
    // block (node-pair) CSR: row A holds the sorted neighbour nodes B
    std::vector<int64_t> bptr;
    std::vector<int32_t> bcol;
    std::vector<int32_t> kdiag;  // position of A in its own block row
    // slot[k*nn + b]: position, in block row A, of local node b of incidence k of A
    std::vector<int16_t> slot;
    int nbmax = 0;  // largest block row
    int64_t nblock() const { return (int64_t)bcol.size(); }
    int64_t nupper() const;  // blocks with A <= B
};

// Returns false (with msg) when the mesh is inconsistent or too large for 31-bit codes.
bool build_pattern(int nd, int nn, int64_t npoint, int64_t ncell, const int64_t* conn, Pattern& pat,
                   const char** msg);

}  // namespace pms
