// pms_pattern.cpp -- see pms_pattern.h.
#include "pms_pattern.h"

#include <algorithm>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace pms {

namespace {
// sorted, unique neighbour nodes of A (the nodes of its incident cells)
void row_nodes(const Pattern& p, const int64_t* conn, int64_t A, std::vector<int32_t>& cols) {
    cols.clear();
    for (int64_t k = p.inc_ptr[A]; k < p.inc_ptr[A + 1]; k++) {
        const int64_t cell = p.inc[k] / p.nn;
        const int64_t* c = conn + cell * p.nn;
        for (int b = 0; b < p.nn; b++) cols.push_back((int32_t)c[b]);
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
}
}  // namespace

int64_t Pattern::nupper() const {
    int64_t n = 0;
    for (int64_t A = 0; A < npoint; A++)
        for (int64_t k = bptr[A]; k < bptr[A + 1]; k++) n += bcol[k] >= A;
    return n;
}

bool build_pattern(int nd, int nn, int64_t npoint, int64_t ncell, const int64_t* conn, Pattern& p, const char** msg) {
    p.nd = nd;
    p.nn = nn;
    p.npoint = npoint;
    p.ncell = ncell;
    if (npoint >= (int64_t)1 << 31 || ncell * (int64_t)nn >= (int64_t)1 << 31) {
        *msg = "mesh too large for 31-bit gather codes";
        return false;
    }
    for (int64_t i = 0; i < ncell * nn; i++)
        if (conn[i] < 0 || conn[i] >= npoint) {
            *msg = "cell connectivity refers to a point that does not exist";
            return false;
        }
    // node -> incidences (ascending cell because cells are visited in order)
    p.inc_ptr.assign(npoint + 1, 0);
    for (int64_t i = 0; i < ncell * nn; i++) p.inc_ptr[conn[i] + 1]++;
    for (int64_t A = 0; A < npoint; A++) p.inc_ptr[A + 1] += p.inc_ptr[A];
    p.inc.assign(ncell * nn, 0);
    {
        std::vector<int64_t> pos(p.inc_ptr.begin(), p.inc_ptr.end() - 1);
        for (int64_t e = 0; e < ncell; e++)
            for (int a = 0; a < nn; a++) p.inc[pos[conn[e * nn + a]]++] = (int32_t)(e * nn + a);
    }
    // pass 1: block row lengths
    std::vector<int64_t> nb(npoint, 0);
#pragma omp parallel
    {
        std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 256)
        for (int64_t A = 0; A < npoint; A++) {
            row_nodes(p, conn, A, cols);
            nb[A] = (int64_t)cols.size();
        }
    }
    p.bptr.assign(npoint + 1, 0);
    int64_t mx = 0;
    for (int64_t A = 0; A < npoint; A++) {
        p.bptr[A + 1] = p.bptr[A] + nb[A];
        mx = std::max(mx, nb[A]);
    }
    if (mx > 32767) {
        *msg = "a block row of the matrix has more than 32767 node blocks";
        return false;
    }
    p.nbmax = (int)mx;
    p.bcol.assign(p.bptr[npoint], 0);
    p.kdiag.assign(npoint, 0);
    p.slot.assign((size_t)ncell * nn * nn, 0);
    // pass 2: columns, diagonal positions and the slot map
#pragma omp parallel
    {
        std::vector<int32_t> cols;
#pragma omp for schedule(dynamic, 256)
        for (int64_t A = 0; A < npoint; A++) {
            row_nodes(p, conn, A, cols);
            std::copy(cols.begin(), cols.end(), p.bcol.begin() + p.bptr[A]);
            auto it = std::lower_bound(cols.begin(), cols.end(), (int32_t)A);
            p.kdiag[A] = (it != cols.end() && *it == A) ? (int32_t)(it - cols.begin()) : 0;
            for (int64_t k = p.inc_ptr[A]; k < p.inc_ptr[A + 1]; k++) {
                const int64_t cell = p.inc[k] / nn;
                const int64_t* c = conn + cell * nn;
                for (int b = 0; b < nn; b++)
                    p.slot[(size_t)k * nn + b] =
                        (int16_t)(std::lower_bound(cols.begin(), cols.end(), (int32_t)c[b]) - cols.begin());
            }
        }
    }
    // processing order of the direct assembly: within each segment (a maximal cell range that shares
    // no node with the cells outside it), the cells by colour, then by index.  Colours are greedy in
    // ascending cell order (cells that share a node get different colours), so consecutive cells of
    // the order never share a node and a cell's predecessors in any of its rows were processed about
    // one colour class earlier.
    std::vector<int32_t> color((size_t)ncell, 0);
    int ncolor = 0;
    {
        std::vector<int64_t> stamp;  // stamp[k] = c: colour k is taken by a lower neighbour of cell c
        for (int64_t c = 0; c < ncell; c++) {
            for (int a = 0; a < nn; a++) {
                const int64_t A = conn[c * nn + a];
                for (int64_t k = p.inc_ptr[A]; k < p.inc_ptr[A + 1]; k++) {
                    const int64_t c2 = p.inc[k] / nn;
                    if (c2 >= c) break;  // incidences are in ascending cell order
                    const int32_t k2 = color[c2];
                    if ((size_t)k2 >= stamp.size()) stamp.resize((size_t)k2 + 1, -1);
                    stamp[k2] = c;
                }
            }
            int32_t k = 0;
            while ((size_t)k < stamp.size() && stamp[k] == c) k++;
            color[c] = k;
            ncolor = std::max(ncolor, (int)k + 1);
        }
    }
    p.ncolor = ncolor;
    p.order.assign((size_t)ncell, 0);
    std::vector<int64_t> opos((size_t)ncell, 0);
    {
        int64_t reach = -1, s0 = 0;  // highest cell that shares a node with a cell of [s0, c)
        std::vector<int64_t> count;
        auto close = [&](int64_t s, int64_t e) {  // counting sort of [s, e) by colour, stable
            count.assign((size_t)ncolor + 1, 0);
            for (int64_t c = s; c < e; c++) count[color[c] + 1]++;
            for (int k = 0; k < ncolor; k++) count[k + 1] += count[k];
            for (int64_t c = s; c < e; c++) {
                const int64_t pos = s + count[color[c]]++;
                p.order[pos] = (int32_t)c;
                opos[c] = pos;
            }
        };
        for (int64_t c = 0; c < ncell; c++) {
            if (reach < c && c > s0) {
                close(s0, c);
                s0 = c;
            }
            for (int a = 0; a < nn; a++) {
                const int64_t A = conn[c * nn + a];
                reach = std::max(reach, (int64_t)(p.inc[p.inc_ptr[A + 1] - 1] / nn));
            }
        }
        if (ncell > s0) close(s0, ncell);
    }
    // per-cell maps of the direct assembly, in the processing order of each row's cells
    p.cslot.assign((size_t)ncell * nn * nn, 0);
    p.crank.assign((size_t)ncell * nn, 0);
    p.cfirst.assign((size_t)ncell * nn, 0);
#pragma omp parallel
    {
        std::vector<char> seen;  // block columns of row A already touched by earlier cells of A
        std::vector<int64_t> ks;
#pragma omp for schedule(dynamic, 1024)
        for (int64_t A = 0; A < npoint; A++) {
            seen.assign((size_t)(p.bptr[A + 1] - p.bptr[A]), 0);
            ks.clear();
            for (int64_t k = p.inc_ptr[A]; k < p.inc_ptr[A + 1]; k++) ks.push_back(k);
            std::sort(ks.begin(), ks.end(), [&](int64_t x, int64_t y) { return opos[p.inc[x] / nn] < opos[p.inc[y] / nn]; });
            for (size_t r = 0; r < ks.size(); r++) {
                const int64_t k = ks[r];
                const int64_t ca = p.inc[k];  // cell * nn + a
                p.crank[ca] = (int32_t)r | (r + 1 == ks.size() ? CRANK_LAST : 0);
                std::memcpy(&p.cslot[(size_t)ca * nn], &p.slot[(size_t)k * nn], sizeof(int16_t) * nn);
                uint32_t first = 0;
                for (int b = 0; b < nn; b++)
                    if (!seen[p.slot[(size_t)k * nn + b]]) first |= 1u << b;
                for (int b = 0; b < nn; b++) seen[p.slot[(size_t)k * nn + b]] = 1;
                p.cfirst[ca] = first;
            }
        }
    }
    return true;
}

}  // namespace pms
