// pms_pattern.cpp -- see pms_pattern.h.
#include "pms_pattern.h"

#include <algorithm>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace pms {

namespace {
struct Item {
    int32_t B;
    int32_t cell;
    int16_t a, b;
};

// all (B, cell, a, b) for the incidences of node A, sorted by (B, cell)
void row_items(const Pattern& p, const int64_t* conn, int64_t A, std::vector<Item>& it) {
    it.clear();
    for (int64_t k = p.inc_ptr[A]; k < p.inc_ptr[A + 1]; k++) {
        int32_t code = p.inc[k];
        int32_t cell = code / p.nn;
        int16_t a = (int16_t)(code % p.nn);
        const int64_t* c = conn + (int64_t)cell * p.nn;
        for (int b = 0; b < p.nn; b++) it.push_back(Item{(int32_t)c[b], cell, a, (int16_t)b});
    }
    std::sort(it.begin(), it.end(), [](const Item& x, const Item& y) {
        if (x.B != y.B) return x.B < y.B;
        if (x.cell != y.cell) return x.cell < y.cell;
        if (x.a != y.a) return x.a < y.a;
        return x.b < y.b;
    });
}
}  // namespace

bool build_pattern(int nd, int nn, int64_t npoint, int64_t ncell, const int64_t* conn, Pattern& p, const char** msg) {
    p.nd = nd;
    p.nn = nn;
    p.npair = nn * (nn + 1) / 2;
    p.npoint = npoint;
    p.ncell = ncell;
    if (npoint >= (int64_t)1 << 31 || ncell * (int64_t)nn >= (int64_t)1 << 31 ||
        ncell * (int64_t)p.npair >= (int64_t)1 << 31) {
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
    // pass 1: counts per block row
    std::vector<int64_t> nb(npoint, 0), nu(npoint, 0), nc(npoint, 0);
#pragma omp parallel
    {
        std::vector<Item> it;
#pragma omp for schedule(dynamic, 256)
        for (int64_t A = 0; A < npoint; A++) {
            row_items(p, conn, A, it);
            int64_t cb = 0, cu = 0, cc = 0;
            for (size_t k = 0; k < it.size(); k++) {
                bool first = (k == 0 || it[k].B != it[k - 1].B);
                if (first) cb++;
                if (it[k].B >= A) {
                    if (first) cu++;
                    cc++;
                }
            }
            nb[A] = cb;
            nu[A] = cu;
            nc[A] = cc;
        }
    }
    p.bptr.assign(npoint + 1, 0);
    std::vector<int64_t> uptr(npoint + 1, 0), cptr(npoint + 1, 0);
    for (int64_t A = 0; A < npoint; A++) {
        p.bptr[A + 1] = p.bptr[A] + nb[A];
        uptr[A + 1] = uptr[A] + nu[A];
        cptr[A + 1] = cptr[A] + nc[A];
    }
    p.bcol.assign(p.bptr[npoint], 0);
    int64_t NU = uptr[npoint], NC = cptr[npoint];
    p.u_row.assign(NU, 0);
    p.u_kab.assign(NU, 0);
    p.u_kba.assign(NU, 0);
    p.u_col.assign(NU, 0);
    p.u_cptr.assign(NU + 1, 0);
    p.u_contrib.assign(NC, 0);
    // pass 2: fill
#pragma omp parallel
    {
        std::vector<Item> it;
#pragma omp for schedule(dynamic, 256)
        for (int64_t A = 0; A < npoint; A++) {
            row_items(p, conn, A, it);
            int64_t kb = p.bptr[A] - 1, ku = uptr[A] - 1, kc = cptr[A];
            for (size_t k = 0; k < it.size(); k++) {
                const Item& x = it[k];
                bool first = (k == 0 || x.B != it[k - 1].B);
                if (first) p.bcol[++kb] = x.B;
                if (x.B >= A) {
                    if (first) {
                        ++ku;
                        p.u_row[ku] = (int32_t)A;
                        p.u_col[ku] = x.B;
                        p.u_kab[ku] = (int32_t)(kb - p.bptr[A]);
                        p.u_cptr[ku] = kc;
                    }
                    int a = x.a, b = x.b;
                    bool tr = a > b;
                    int q = tr ? pair_index(nn, b, a) : pair_index(nn, a, b);
                    uint32_t code = (uint32_t)((int64_t)x.cell * p.npair + q) | (tr ? 0x80000000u : 0u);
                    p.u_contrib[kc++] = (int32_t)code;
                }
            }
        }
    }
    p.u_cptr[NU] = NC;
    p.uptr = uptr;
    p.kdiag.assign(npoint, 0);
    for (int64_t A = 0; A < npoint; A++) p.kdiag[A] = (uptr[A + 1] > uptr[A]) ? p.u_kab[uptr[A]] : 0;
    // position of A in block row B
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < NU; u++) {
        int32_t A = p.u_row[u], B = p.u_col[u];
        const int32_t* b0 = p.bcol.data() + p.bptr[B];
        const int32_t* b1 = p.bcol.data() + p.bptr[B + 1];
        p.u_kba[u] = (int32_t)(std::lower_bound(b0, b1, A) - b0);
    }
    return true;
}

}  // namespace pms
