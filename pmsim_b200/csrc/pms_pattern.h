// pms_pattern.h -- CSR pattern of the global matrix and the deterministic gather maps.
//
// The reference assembles K as COO triplets with duplicates in cell order and lets the
// sparse solver sum them (src/base/assembly.rs:70-139, src/fem/linear_system.rs:132-164).
// Here the pattern is built once per mesh: for every node pair (A, B) with A <= B that shares
// a cell ("upper block"), the list of element blocks that contribute to it, in ascending cell
// order.  The assembly kernel then owns each upper block with one thread, sums the list in that
// fixed order (no atomics) and writes both K_AB and K_BA = K_AB^T, so the result is the same bits
// on every run.
#pragma once
#include <cstdint>
#include <vector>

namespace pms {

struct Pattern {
    int nd = 0, nn = 0, npair = 0;
    int64_t npoint = 0, ncell = 0;
    // node -> (cell*nn + local) incidences, ascending cell
    std::vector<int64_t> inc_ptr;
    std::vector<int32_t> inc;
    // block (node-pair) CSR: row A holds the sorted neighbour nodes B
    std::vector<int64_t> bptr;
    std::vector<int32_t> bcol;
    // upper blocks (A <= B)
    std::vector<int32_t> u_row;   // A
    std::vector<int32_t> u_kab;   // position of B in block row A
    std::vector<int32_t> u_kba;   // position of A in block row B
    std::vector<int32_t> u_col;   // B
    std::vector<int64_t> u_cptr;  // contributions of upper block u: [u_cptr[u], u_cptr[u+1])
    std::vector<int32_t> u_contrib;  // (cell*npair + pair) | transpose<<31
    std::vector<int64_t> uptr;       // upper blocks of block row A: [uptr[A], uptr[A+1])
    std::vector<int32_t> kdiag;      // position of A in its own block row (first upper block)
    int64_t nblock() const { return (int64_t)bcol.size(); }
    int64_t nupper() const { return (int64_t)u_row.size(); }
};

// pair index of local nodes (a <= b): rows of the upper triangle of the node-pair matrix
inline int pair_index(int nn, int a, int b) { return a * nn - a * (a - 1) / 2 + (b - a); }

// Returns false (with msg) when the mesh is inconsistent or too large for 31-bit codes.
bool build_pattern(int nd, int nn, int64_t npoint, int64_t ncell, const int64_t* conn, Pattern& pat,
                   const char** msg);

}  // namespace pms
