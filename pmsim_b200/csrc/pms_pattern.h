// pms_pattern.h -- CSR pattern of the global matrix and the deterministic gather maps.
//
// The reference assembles K as COO triplets with duplicates in cell order and lets the
// sparse solver sum them (src/base/assembly.rs:70-139, src/fem/linear_system.rs:132-164).
// Here the pattern is built once per mesh.  Block row A of K (node A, ND x ND blocks) is the sum,
// over the cells incident to A, of the node-row slab (a, all b) of each cell's element matrix, where
// a is A's local index in the cell.  Two assemblies use it, both with the same bits on every run
// (every node-pair block summed over its cells in a fixed order):
//  * direct: the element kernel takes the cells in a processing order (order: colour classes, so
//    that cells taken one after another share no node) and adds cell c's slab a into row A once
//    the cells before c, in that order, among A's cells have added theirs (rank[c*nn + a] = c's
//    position; a ticket per row counts the slabs added), at the columns cslot[(c*nn + a)*nn + b];
//    a block's first contribution (cfirst) is stored, the later ones are added;
//  * gather: a kernel owns one block row and adds the slabs of the cells' dense element matrices in
//    ascending cell order (slot[k*nn + b]: where local node b of incidence k of A lands in the row).
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
    // per cell (direct assembly): cslot[(c*nn + a)*nn + b] = position, in block row conn[c][a], of
    // node b; crank[c*nn + a] = position of c among the cells of node conn[c][a] (bits 0..29),
    // bit 30 set when c is the last of them
    std::vector<int16_t> cslot;
    std::vector<int32_t> crank;
    // cfirst[c*nn + a] bit b: c is the first cell (in the processing order) that holds both conn[c][a]
    // and conn[c][b], so it stores the first contribution of block (conn[a], conn[b]) (and of its
    // mirror); later cells add to it
    std::vector<uint32_t> cfirst;
    // processing order of the direct assembly (order[k] = k-th cell): within each segment of cells
    // that shares no node with the rest, by greedy colour then index; crank and cfirst follow it
    std::vector<int32_t> order;
    int ncolor = 0;
    int nbmax = 0;  // largest block row
    int64_t nblock() const { return (int64_t)bcol.size(); }
    int64_t nupper() const;  // blocks with A <= B
};

// Returns false (with msg) when the mesh is inconsistent or too large for 31-bit codes.
bool build_pattern(int nd, int nn, int64_t npoint, int64_t ncell, const int64_t* conn, Pattern& pat,
                   const char** msg);

constexpr int32_t CRANK_LAST = 1 << 30;
constexpr int32_t CRANK_MASK = CRANK_LAST - 1;

}  // namespace pms
