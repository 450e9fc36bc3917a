// pms_oracle.cpp -- CPU restatement of pmsim 0.3.0's implicit solid hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests, the smoke check
// and the CPU-baseline leg of bench.py load it as the checker (or as the timed CPU
// restatement).  The product path (pmsim_b200, libpms_b200.so) never links or calls it.
//
// What it restates (reference file:line, paths inside the pmsim project):
//   * VonMises::update_stress / stiffness        src/material/von_mises.rs:124-226
//   * LinearElastic::update_stress / stiffness   src/material/linear_elastic.rs:49-71
//   * LocalState (elastic, int_vars=[z,lambda], stress)  src/material/local_state.rs:9-44
//   * calculate_strain (2D plane strain, 3D)     src/base/calculate_strain.rs:18-60
//   * ElementSolid::calc_f_int / calc_jacobian / update_secondary_values
//                                                src/fem/element_solid.rs:124-224
//   * assemble_vector / assemble_matrix (COO with duplicates, symmetry check)
//                                                src/base/assembly.rs:38-139
//   * Elements loops over cells                  src/fem/elements.rs:132-205
// Third-party arithmetic the reference delegates to un-vendored crates (gemlab,
// russell_tensor; path dependencies with no lockfile, so their versions are unpinned)
// is restated from the textbook mathematics:
//   * Lagrange / serendipity shape functions of Tri3/Tri6/Qua4/Qua8/Qua9/Tet4/Tet10/
//     Hex8/Hex20 (Zienkiewicz & Taylor, The Finite Element Method, Vol. 1, ch. 6),
//   * tensor-product Gauss-Legendre rules on [-1,1]^d and the standard interior rules of
//     the reference triangle/tetrahedron (Strang & Fix; Hammer-Stroud),
//   * Mandel (Kelvin) notation for symmetric second/fourth order tensors,
//     sigma = [xx, yy, zz, sqrt2*xy, sqrt2*yz, sqrt2*xz] (de Souza Neto, Peric & Owen,
//     Computational Methods for Plasticity, 2008).
// Node ordering (corners, then mid-edges 0-1,1-2,2-3,3-0 for Qua8; bottom, top, vertical
// mid-edges for Hex20) is the one pinned by the reference's mesh files
// (data/results/artificial/*.msh, src/base/sample_meshes.rs:541-625).
// Parity pins: the inline KATs of src/material/von_mises.rs:324-480 and the SPO/HYPLAS
// golden runs (data/spo/*.json) replayed by oracle/driver.py (tests/test_oracle_*.py).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <numeric>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum Kind { TRI3 = 0, TRI6 = 1, QUA4 = 2, QUA8 = 3, QUA9 = 4, TET4 = 5, TET10 = 6, HEX8 = 7, HEX20 = 8,
            TRI10 = 9, TRI15 = 10 };
constexpr int NKIND = 11;

const double SQRT2 = 1.4142135623730951;
const double SQRT_2_BY_3 = 0.816496580927726;   // sqrt(2/3)
const double F_TOL = 1e-6;                       // src/material/von_mises.rs:23

int kind_nnode(int k) {
    static const int n[] = {3, 6, 4, 8, 9, 4, 10, 8, 20, 10, 15};
    return (k >= 0 && k < NKIND) ? n[k] : -1;
}
int kind_ndim(int k) { return (k <= QUA9 || k == TRI10 || k == TRI15) ? 2 : 3; }

int default_ngauss(int k) {
    static const int n[] = {3, 3, 4, 9, 9, 4, 4, 8, 27, 6, 12};
    return (k >= 0 && k < NKIND) ? n[k] : -1;
}

// ---------------------------------------------------------------- Gauss rules
void legendre_1d(int n, double* x, double* w) {
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; }
    else if (n == 2) { double a = 1.0 / std::sqrt(3.0); x[0] = -a; x[1] = a; w[0] = w[1] = 1.0; }
    else { double a = std::sqrt(3.0 / 5.0); x[0] = -a; x[1] = 0.0; x[2] = a;
           w[0] = 5.0 / 9.0; w[1] = 8.0 / 9.0; w[2] = 5.0 / 9.0; }
}

// Tensor-product rule, x varies fastest, then y, then z.
int gauss_rule(int kind, int ngauss, double* ksi /*ngauss*3*/, double* w) {
    int nd = kind_ndim(kind);
    bool simplex = (kind == TRI3 || kind == TRI6 || kind == TET4 || kind == TET10 || kind == TRI10 || kind == TRI15);
    if (!simplex) {
        int n1 = 0;
        if (nd == 2) { if (ngauss == 1) n1 = 1; else if (ngauss == 4) n1 = 2; else if (ngauss == 9) n1 = 3; }
        else { if (ngauss == 1) n1 = 1; else if (ngauss == 8) n1 = 2; else if (ngauss == 27) n1 = 3; }
        if (n1 == 0) return -1;
        double x[3], ww[3];
        legendre_1d(n1, x, ww);
        int p = 0;
        int nz = (nd == 3) ? n1 : 1;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < n1; j++)
                for (int i = 0; i < n1; i++) {
                    ksi[3 * p + 0] = x[i];
                    ksi[3 * p + 1] = x[j];
                    ksi[3 * p + 2] = (nd == 3) ? x[k] : 0.0;
                    w[p] = ww[i] * ww[j] * ((nd == 3) ? ww[k] : 1.0);
                    p++;
                }
        return p;
    }
    if (nd == 2) {
        if (ngauss == 1) { ksi[0] = 1.0 / 3.0; ksi[1] = 1.0 / 3.0; ksi[2] = 0; w[0] = 0.5; return 1; }
        if (ngauss == 3) {
            const double a = 1.0 / 6.0, b = 2.0 / 3.0;
            double pts[3][2] = {{a, a}, {b, a}, {a, b}};
            for (int p = 0; p < 3; p++) { ksi[3*p] = pts[p][0]; ksi[3*p+1] = pts[p][1]; ksi[3*p+2] = 0; w[p] = 1.0 / 6.0; }
            return 3;
        }
        // symmetric triangle rules of Dunavant (1985): orbits of barycentric points (a, a, 1-2a), the
        // centroid, and (a, b, 1-a-b) with its six permutations; weights for unit area, times 1/2 here
        struct Orbit { int kind; double w, a, b; };  // kind 1: centroid, 3: (a,a,1-2a), 6: (a,b,c)
        Orbit orb[3];
        int norb = 0;
        if (ngauss == 6) {  // degree 4
            orb[0] = {3, 0.223381589678011, 0.445948490915965, 0};
            orb[1] = {3, 0.109951743655322, 0.091576213509771, 0};
            norb = 2;
        } else if (ngauss == 7) {  // degree 5 (closed form)
            const double r15 = std::sqrt(15.0);
            orb[0] = {1, 0.225, 1.0 / 3.0, 0};
            orb[1] = {3, (155.0 + r15) / 1200.0, (6.0 + r15) / 21.0, 0};
            orb[2] = {3, (155.0 - r15) / 1200.0, (6.0 - r15) / 21.0, 0};
            norb = 3;
        } else if (ngauss == 12) {  // degree 6
            orb[0] = {3, 0.116786275726379, 0.249286745170910, 0};
            orb[1] = {3, 0.050844906370207, 0.063089014491502, 0};
            orb[2] = {6, 0.082851075618374, 0.053145049844817, 0.310352451033784};
            norb = 3;
        } else {
            return -1;
        }
        int p = 0;
        for (int io = 0; io < norb; io++) {
            const Orbit& o = orb[io];
            double pts[6][2];
            int n = 0;
            if (o.kind == 1) { pts[0][0] = o.a; pts[0][1] = o.a; n = 1; }
            else if (o.kind == 3) {
                const double c = 1.0 - 2.0 * o.a;
                double q[3][2] = {{o.a, o.a}, {c, o.a}, {o.a, c}};
                for (int i = 0; i < 3; i++) { pts[i][0] = q[i][0]; pts[i][1] = q[i][1]; }
                n = 3;
            } else {
                const double c = 1.0 - o.a - o.b;
                double q[6][2] = {{o.a, o.b}, {o.b, o.a}, {o.b, c}, {c, o.b}, {c, o.a}, {o.a, c}};
                for (int i = 0; i < 6; i++) { pts[i][0] = q[i][0]; pts[i][1] = q[i][1]; }
                n = 6;
            }
            for (int i = 0; i < n; i++, p++) {
                ksi[3 * p] = pts[i][0];
                ksi[3 * p + 1] = pts[i][1];
                ksi[3 * p + 2] = 0.0;
                w[p] = 0.5 * o.w;
            }
        }
        return p;
    }
    if (ngauss == 1) { ksi[0] = ksi[1] = ksi[2] = 0.25; w[0] = 1.0 / 6.0; return 1; }
    if (ngauss == 4) {
        const double a = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, b = (5.0 - std::sqrt(5.0)) / 20.0;
        double pts[4][3] = {{b, b, b}, {a, b, b}, {b, a, b}, {b, b, a}};
        for (int p = 0; p < 4; p++) { for (int d = 0; d < 3; d++) ksi[3*p+d] = pts[p][d]; w[p] = 1.0 / 24.0; }
        return 4;
    }
    return -1;
}

// ---------------------------------------------------------------- shape functions
// Complete Lagrange triangle of order n in area coordinates L0 = 1 - r - s, L1 = r, L2 = s: the node
// at barycentric position (i, j, k)/n has N = P_i(L0) P_j(L1) P_k(L2), P_a(L) = prod_{q<a} (nL - q)/(q+1)
// (Silvester's formula; Zienkiewicz & Taylor Vol. 1, sec. 6.6).  Node order: corners; for n = 4 the
// mid-edge nodes of edges 0-1, 1-2, 2-0; then per edge the node nearer its first corner and the one
// nearer its second; then the interior nodes.
const int TRI10_IJK[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {1, 2, 0},
                              {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {2, 0, 1}, {1, 1, 1}};
const int TRI15_IJK[15][3] = {{4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}, {3, 1, 0}, {1, 3, 0},
                              {0, 3, 1}, {0, 1, 3}, {1, 0, 3}, {3, 0, 1}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};

void silvester(int n, int a, double L, double& P, double& dP) {
    P = 1.0;
    dP = 0.0;
    for (int q = 0; q < a; q++) {
        const double f = (n * L - q) / (q + 1);
        dP = dP * f + P * n / (q + 1);
        P *= f;
    }
}

void lagrange_triangle(int n, int nn, const int (*ijk)[3], double r, double s, double* N, double* dN) {
    const double L0 = 1.0 - r - s;
    for (int m = 0; m < nn; m++) {
        double P0, d0, P1, d1, P2, d2;
        silvester(n, ijk[m][0], L0, P0, d0);
        silvester(n, ijk[m][1], r, P1, d1);
        silvester(n, ijk[m][2], s, P2, d2);
        N[m] = P0 * P1 * P2;
        dN[2 * m] = -d0 * P1 * P2 + P0 * d1 * P2;
        dN[2 * m + 1] = -d0 * P1 * P2 + P0 * P1 * d2;
    }
}

// N[m], dN[m*nd + j] = dN_m/dksi_j
void shape(int kind, const double* k, double* N, double* dN) {
    const double r = k[0], s = k[1], t = k[2];
    switch (kind) {
    case TRI10:
        lagrange_triangle(3, 10, TRI10_IJK, r, s, N, dN);
        break;
    case TRI15:
        lagrange_triangle(4, 15, TRI15_IJK, r, s, N, dN);
        break;
    case TRI3:
        N[0] = 1 - r - s; N[1] = r; N[2] = s;
        dN[0] = -1; dN[1] = -1; dN[2] = 1; dN[3] = 0; dN[4] = 0; dN[5] = 1;
        break;
    case TRI6: {
        double L0 = 1 - r - s, L1 = r, L2 = s;
        N[0] = L0 * (2 * L0 - 1); N[1] = L1 * (2 * L1 - 1); N[2] = L2 * (2 * L2 - 1);
        N[3] = 4 * L0 * L1; N[4] = 4 * L1 * L2; N[5] = 4 * L2 * L0;
        // dL0 = (-1,-1), dL1 = (1,0), dL2 = (0,1)
        double d0 = 4 * L0 - 1, d1 = 4 * L1 - 1, d2 = 4 * L2 - 1;
        dN[0] = -d0; dN[1] = -d0;
        dN[2] = d1;  dN[3] = 0;
        dN[4] = 0;   dN[5] = d2;
        dN[6] = 4 * (L0 - L1); dN[7] = -4 * L1;
        dN[8] = 4 * L2;        dN[9] = 4 * L1;
        dN[10] = -4 * L2;      dN[11] = 4 * (L0 - L2);
        break;
    }
    case QUA4: {
        static const double xi[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
        for (int m = 0; m < 4; m++) {
            double a = xi[m][0], b = xi[m][1];
            N[m] = (1 + a * r) * (1 + b * s) / 4.0;
            dN[2 * m] = a * (1 + b * s) / 4.0;
            dN[2 * m + 1] = b * (1 + a * r) / 4.0;
        }
        break;
    }
    case QUA8: {
        static const double xi[8][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}};
        for (int m = 0; m < 8; m++) {
            double a = xi[m][0], b = xi[m][1];
            if (m < 4) {
                N[m] = (1 + a * r) * (1 + b * s) * (a * r + b * s - 1) / 4.0;
                dN[2 * m] = a * (1 + b * s) * (2 * a * r + b * s) / 4.0;
                dN[2 * m + 1] = b * (1 + a * r) * (a * r + 2 * b * s) / 4.0;
            } else if (a == 0) {
                N[m] = (1 - r * r) * (1 + b * s) / 2.0;
                dN[2 * m] = -r * (1 + b * s);
                dN[2 * m + 1] = b * (1 - r * r) / 2.0;
            } else {
                N[m] = (1 + a * r) * (1 - s * s) / 2.0;
                dN[2 * m] = a * (1 - s * s) / 2.0;
                dN[2 * m + 1] = -s * (1 + a * r);
            }
        }
        break;
    }
    case QUA9: {
        // 1D quadratic Lagrange at -1, 0, +1
        auto l = [](int i, double x) { return i == 0 ? x * (x - 1) / 2.0 : (i == 1 ? 1 - x * x : x * (x + 1) / 2.0); };
        auto dl = [](int i, double x) { return i == 0 ? x - 0.5 : (i == 1 ? -2 * x : x + 0.5); };
        static const int ij[9][2] = {{0, 0}, {2, 0}, {2, 2}, {0, 2}, {1, 0}, {2, 1}, {1, 2}, {0, 1}, {1, 1}};
        for (int m = 0; m < 9; m++) {
            int i = ij[m][0], j = ij[m][1];
            N[m] = l(i, r) * l(j, s);
            dN[2 * m] = dl(i, r) * l(j, s);
            dN[2 * m + 1] = l(i, r) * dl(j, s);
        }
        break;
    }
    case TET4:
        N[0] = 1 - r - s - t; N[1] = r; N[2] = s; N[3] = t;
        for (int j = 0; j < 3; j++) dN[j] = -1;
        dN[3] = 1; dN[4] = 0; dN[5] = 0;
        dN[6] = 0; dN[7] = 1; dN[8] = 0;
        dN[9] = 0; dN[10] = 0; dN[11] = 1;
        break;
    case TET10: {
        double L[4] = {1 - r - s - t, r, s, t};
        static const double dL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        static const int ed[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
        for (int m = 0; m < 4; m++) {
            N[m] = L[m] * (2 * L[m] - 1);
            for (int j = 0; j < 3; j++) dN[3 * m + j] = (4 * L[m] - 1) * dL[m][j];
        }
        for (int e = 0; e < 6; e++) {
            int a = ed[e][0], b = ed[e][1], m = 4 + e;
            N[m] = 4 * L[a] * L[b];
            for (int j = 0; j < 3; j++) dN[3 * m + j] = 4 * (dL[a][j] * L[b] + L[a] * dL[b][j]);
        }
        break;
    }
    case HEX8: {
        static const double xi[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                        {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
        for (int m = 0; m < 8; m++) {
            double a = xi[m][0], b = xi[m][1], c = xi[m][2];
            N[m] = (1 + a * r) * (1 + b * s) * (1 + c * t) / 8.0;
            dN[3 * m] = a * (1 + b * s) * (1 + c * t) / 8.0;
            dN[3 * m + 1] = b * (1 + a * r) * (1 + c * t) / 8.0;
            dN[3 * m + 2] = c * (1 + a * r) * (1 + b * s) / 8.0;
        }
        break;
    }
    case HEX20: {
        static const double xi[20][3] = {
            {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
            {0, -1, -1},  {1, 0, -1},  {0, 1, -1}, {-1, 0, -1}, {0, -1, 1},  {1, 0, 1},  {0, 1, 1}, {-1, 0, 1},
            {-1, -1, 0},  {1, -1, 0},  {1, 1, 0},  {-1, 1, 0}};
        for (int m = 0; m < 20; m++) {
            double a = xi[m][0], b = xi[m][1], c = xi[m][2];
            if (m < 8) {
                double ar = 1 + a * r, bs = 1 + b * s, ct = 1 + c * t, q = a * r + b * s + c * t - 2;
                N[m] = ar * bs * ct * q / 8.0;
                dN[3 * m] = a * bs * ct * (q + ar) / 8.0;
                dN[3 * m + 1] = b * ar * ct * (q + bs) / 8.0;
                dN[3 * m + 2] = c * ar * bs * (q + ct) / 8.0;
            } else if (a == 0) {
                double bs = 1 + b * s, ct = 1 + c * t;
                N[m] = (1 - r * r) * bs * ct / 4.0;
                dN[3 * m] = -2 * r * bs * ct / 4.0;
                dN[3 * m + 1] = (1 - r * r) * b * ct / 4.0;
                dN[3 * m + 2] = (1 - r * r) * bs * c / 4.0;
            } else if (b == 0) {
                double ar = 1 + a * r, ct = 1 + c * t;
                N[m] = ar * (1 - s * s) * ct / 4.0;
                dN[3 * m] = a * (1 - s * s) * ct / 4.0;
                dN[3 * m + 1] = -2 * s * ar * ct / 4.0;
                dN[3 * m + 2] = ar * (1 - s * s) * c / 4.0;
            } else {
                double ar = 1 + a * r, bs = 1 + b * s;
                N[m] = ar * bs * (1 - t * t) / 4.0;
                dN[3 * m] = a * bs * (1 - t * t) / 4.0;
                dN[3 * m + 1] = ar * b * (1 - t * t) / 4.0;
                dN[3 * m + 2] = -2 * t * ar * bs / 4.0;
            }
        }
        break;
    }
    }
}

// ---------------------------------------------------------------- Mandel helpers
// I = [1,1,1,0,0,0];  Psd = Id - I(x)I/3 (symmetric deviatoric projector)
inline double Ivec(int i) { return i < 3 ? 1.0 : 0.0; }
inline double Psd(int i, int j) {
    if (i < 3 && j < 3) return (i == j) ? 2.0 / 3.0 : -1.0 / 3.0;
    return (i == j) ? 1.0 : 0.0;
}
inline double sigma_m(const double* v) { return (v[0] + v[1] + v[2]) / 3.0; }
inline double sigma_d(const double* v, int nc) {
    double m = sigma_m(v), s2 = 0;
    for (int i = 0; i < nc; i++) { double s = v[i] - (i < 3 ? m : 0.0); s2 += s * s; }
    return std::sqrt(1.5 * s2);  // sqrt(3 J2), J2 = s:s/2
}

struct Params { double young, poisson, hh, z_ini; };

void bulk_shear(const Params& p, double& kk, double& gg) {
    kk = p.young / (3.0 * (1.0 - 2.0 * p.poisson));
    gg = p.young / (2.0 * (1.0 + p.poisson));
}

// Hooke's modulus in Mandel form (plane strain uses the 4x4 top-left block)
void elastic_modulus(const Params& p, int nc, double* dd) {
    double c = p.young / ((1.0 + p.poisson) * (1.0 - 2.0 * p.poisson));
    for (int i = 0; i < nc * nc; i++) dd[i] = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) dd[i * nc + j] = (i == j) ? c * (1.0 - p.poisson) : c * p.poisson;
    for (int i = 3; i < nc; i++) dd[i * nc + i] = c * (1.0 - 2.0 * p.poisson);
}

// Plane-stress Hooke modulus (2D, Mandel xx, yy, zz, xy): c = E/(1-nu^2) on the in-plane normal
// block, zz row and column zero, shear c(1-nu) = 2G (russell_tensor LinElasticity with plane_stress,
// used by src/material/linear_elastic.rs:17).
void elastic_modulus_plane_stress(const Params& p, double* dd) {
    double c = p.young / (1.0 - p.poisson * p.poisson);
    for (int i = 0; i < 16; i++) dd[i] = 0;
    dd[0] = dd[5] = c;
    dd[1] = dd[4] = c * p.poisson;
    dd[15] = c * (1.0 - p.poisson);
}

// model: 0 = LinearElastic, 1 = VonMises, 2 = LinearElastic in plane stress (2D).
// ivs = [z, lambda]. returns 0 ok, else error code
//   2: "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)"
//   3: "von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)"
int model_update_stress(int model, const Params& p, int nc, double* sig, double* ivs, uint8_t* elastic,
                        const double* deps) {
    double dd[36];
    if (model == 2) elastic_modulus_plane_stress(p, dd);
    else elastic_modulus(p, nc, dd);
    if (model == 0 || model == 2) {  // src/material/linear_elastic.rs:61-71
        double ds[6];
        for (int i = 0; i < nc; i++) { ds[i] = 0; for (int j = 0; j < nc; j++) ds[i] += dd[i * nc + j] * deps[j]; }
        for (int i = 0; i < nc; i++) sig[i] += ds[i];
        return 0;
    }
    // src/material/von_mises.rs:170-226
    *elastic = 1;
    ivs[1] = 0.0;
    double ds[6];
    for (int i = 0; i < nc; i++) { ds[i] = 0; for (int j = 0; j < nc; j++) ds[i] += dd[i * nc + j] * deps[j]; }
    for (int i = 0; i < nc; i++) sig[i] += ds[i];
    double f_trial = sigma_d(sig, nc) - ivs[0];
    if (f_trial / p.z_ini <= F_TOL) return 0;
    double kk, gg;
    bulk_shear(p, kk, gg);
    double sm = sigma_m(sig), sd_trial = sigma_d(sig, nc);
    double lambda = f_trial / (3.0 * gg + p.hh);
    double beta = 1.0 - lambda * 3.0 * gg / sd_trial;
    double s[6];
    for (int i = 0; i < nc; i++) s[i] = sig[i] - (i < 3 ? sm : 0.0);
    for (int i = 0; i < nc; i++) sig[i] = sm * Ivec(i) + beta * s[i];
    if (sigma_d(sig, nc) < 1e-10) return 2;
    ivs[0] += p.hh * lambda;
    *elastic = 0;
    ivs[1] = lambda;
    return 0;
}

int model_stiffness(int model, const Params& p, int nc, const double* sig, const double* ivs, uint8_t elastic,
                    double* dd) {
    if (model == 2) { elastic_modulus_plane_stress(p, dd); return 0; }
    if (model == 0 || elastic) { elastic_modulus(p, nc, dd); return 0; }
    // src/material/von_mises.rs:124-167
    double kk, gg;
    bulk_shear(p, kk, gg);
    double lambda = ivs[1];
    double sm = sigma_m(sig);
    double s[6];
    for (int i = 0; i < nc; i++) s[i] = sig[i] - (i < 3 ? sm : 0.0);
    double sd = sigma_d(sig, nc);
    double sd_trial = sd + lambda * 3.0 * gg;
    double norm_s = sd * SQRT_2_BY_3;
    if (norm_s < 1e-10) return 3;
    double d = 3.0 * gg + p.hh;
    double a = 2.0 * gg * (1.0 - lambda * 3.0 * gg / sd_trial);
    double b = 6.0 * gg * gg * (lambda / sd_trial - 1.0 / d) / (norm_s * norm_s);
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < nc; j++) dd[i * nc + j] = a * Psd(i, j) + b * s[i] * s[j] + kk * Ivec(i) * Ivec(j);
    return 0;
}

// ---------------------------------------------------------------- element geometry
struct IpGeo { double det; double G[20 * 3]; double N[20]; };

// returns 0 ok, 4 = non-positive Jacobian determinant
int ip_geometry(int kind, const double* X /*nnode*nd*/, const double* ksi, IpGeo& g) {
    int nn = kind_nnode(kind), nd = kind_ndim(kind);
    double dN[20 * 3];
    shape(kind, ksi, g.N, dN);
    double J[9] = {0};
    for (int m = 0; m < nn; m++)
        for (int i = 0; i < nd; i++)
            for (int j = 0; j < nd; j++) J[i * nd + j] += X[m * nd + i] * dN[m * nd + j];
    double Ji[9];
    if (nd == 2) {
        g.det = J[0] * J[3] - J[1] * J[2];
        if (!(g.det > 0)) return 4;
        Ji[0] = J[3] / g.det; Ji[1] = -J[1] / g.det; Ji[2] = -J[2] / g.det; Ji[3] = J[0] / g.det;
    } else {
        g.det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) + J[2] * (J[3] * J[7] - J[4] * J[6]);
        if (!(g.det > 0)) return 4;
        Ji[0] = (J[4] * J[8] - J[5] * J[7]) / g.det;
        Ji[1] = (J[2] * J[7] - J[1] * J[8]) / g.det;
        Ji[2] = (J[1] * J[5] - J[2] * J[4]) / g.det;
        Ji[3] = (J[5] * J[6] - J[3] * J[8]) / g.det;
        Ji[4] = (J[0] * J[8] - J[2] * J[6]) / g.det;
        Ji[5] = (J[2] * J[3] - J[0] * J[5]) / g.det;
        Ji[6] = (J[3] * J[7] - J[4] * J[6]) / g.det;
        Ji[7] = (J[1] * J[6] - J[0] * J[7]) / g.det;
        Ji[8] = (J[0] * J[4] - J[1] * J[3]) / g.det;
    }
    // G[m][i] = sum_j dN[m][j] * Jinv[j][i]
    for (int m = 0; m < nn; m++)
        for (int i = 0; i < nd; i++) {
            double v = 0;
            for (int j = 0; j < nd; j++) v += dN[m * nd + j] * Ji[j * nd + i];
            g.G[m * nd + i] = v;
        }
    return 0;
}

// Mandel B matrix, nc x (nn*nd), row-major
void b_matrix(int nn, int nd, const double* G, double* B) {
    int nc = 2 * nd, ne = nn * nd;
    for (int i = 0; i < nc * ne; i++) B[i] = 0;
    for (int m = 0; m < nn; m++) {
        if (nd == 2) {
            double gx = G[2 * m], gy = G[2 * m + 1];
            B[0 * ne + 2 * m] = gx;
            B[1 * ne + 2 * m + 1] = gy;
            B[3 * ne + 2 * m] = gy / SQRT2;
            B[3 * ne + 2 * m + 1] = gx / SQRT2;
        } else {
            double gx = G[3 * m], gy = G[3 * m + 1], gz = G[3 * m + 2];
            B[0 * ne + 3 * m] = gx;
            B[1 * ne + 3 * m + 1] = gy;
            B[2 * ne + 3 * m + 2] = gz;
            B[3 * ne + 3 * m] = gy / SQRT2; B[3 * ne + 3 * m + 1] = gx / SQRT2;
            B[4 * ne + 3 * m + 1] = gz / SQRT2; B[4 * ne + 3 * m + 2] = gy / SQRT2;
            B[5 * ne + 3 * m] = gz / SQRT2; B[5 * ne + 3 * m + 2] = gx / SQRT2;
        }
    }
}

struct ElemCtx {
    int kind, nn, nd, nc, ngauss;
    double ksi[27 * 3], w[27];
    double thickness;
    bool axisym;  // 2D axisymmetric idealization (x = radius): weight |J| w r, hoop strain u_r / r
};

// Integration weight of an IP: |J| w t, or |J| w r in the axisymmetric idealization (r = sum N_m x_m,
// gemlab's integrators with args.axisymmetric, called by src/fem/element_solid.rs:128,150,171).
inline double ip_coef(const ElemCtx& c, const IpGeo& g, const double* X, int p, double* radius) {
    if (!c.axisym) return g.det * c.w[p] * c.thickness;
    double r = 0.0;
    for (int m = 0; m < c.nn; m++) r += g.N[m] * X[m * 2];
    *radius = r;
    return g.det * c.w[p] * r;
}

// thickness < 0 selects the axisymmetric idealization (2D kinds only)
bool make_ctx(int kind, int ngauss, double thickness, ElemCtx& c) {
    c.kind = kind;
    c.nn = kind_nnode(kind);
    if (c.nn < 0) return false;
    c.nd = kind_ndim(kind);
    c.nc = 2 * c.nd;
    if (ngauss <= 0) ngauss = default_ngauss(kind);
    c.ngauss = gauss_rule(kind, ngauss, c.ksi, c.w);
    c.axisym = thickness < 0.0;
    c.thickness = c.axisym ? 1.0 : thickness;
    if (c.axisym && c.nd != 2) return false;
    return c.ngauss > 0;
}

// f_int: vec_04_tb -- f[m*nd+i] = sum_p sum_j sigma_ij G[m][j] |J| w_p t
int elem_f_int(const ElemCtx& c, const double* X, const double* sig /*ngauss*nc*/, double* f) {
    int ne = c.nn * c.nd;
    for (int i = 0; i < ne; i++) f[i] = 0;
    IpGeo g;
    for (int p = 0; p < c.ngauss; p++) {
        int st = ip_geometry(c.kind, X, c.ksi + 3 * p, g);
        if (st) return st;
        double r = 1.0;
        double coef = ip_coef(c, g, X, p, &r);
        const double* v = sig + p * c.nc;
        double S[3][3];
        S[0][0] = v[0]; S[1][1] = v[1]; S[2][2] = v[2];
        S[0][1] = S[1][0] = v[3] / SQRT2;
        if (c.nd == 3) { S[1][2] = S[2][1] = v[4] / SQRT2; S[0][2] = S[2][0] = v[5] / SQRT2; }
        for (int m = 0; m < c.nn; m++)
            for (int i = 0; i < c.nd; i++) {
                double s = 0;
                for (int j = 0; j < c.nd; j++) s += S[i][j] * g.G[m * c.nd + j];
                if (c.axisym && i == 0) s += v[2] * g.N[m] / r;  // hoop row of B: N/r on u_r
                f[m * c.nd + i] += coef * s;
            }
    }
    return 0;
}

// K: mat_10_bdb -- K = sum_p B^T D B |J| w_p t  (dense, as the reference does it)
int elem_jacobian(const ElemCtx& c, const double* X, int model, const Params& prm, const double* sig,
                  const double* ivs, const uint8_t* elastic, double* K) {
    int ne = c.nn * c.nd;
    for (int i = 0; i < ne * ne; i++) K[i] = 0;
    IpGeo g;
    std::vector<double> B(c.nc * ne), DB(c.nc * ne);
    double dd[36];
    for (int p = 0; p < c.ngauss; p++) {
        int st = ip_geometry(c.kind, X, c.ksi + 3 * p, g);
        if (st) return st;
        st = model_stiffness(model, prm, c.nc, sig + p * c.nc, ivs + 2 * p, elastic[p], dd);
        if (st) return st;
        double r = 1.0;
        double coef = ip_coef(c, g, X, p, &r);
        b_matrix(c.nn, c.nd, g.G, B.data());
        if (c.axisym)
            for (int m = 0; m < c.nn; m++) B[2 * ne + 2 * m] = g.N[m] / r;  // eps_zz = u_r / r
        for (int k = 0; k < c.nc; k++)
            for (int col = 0; col < ne; col++) {
                double s = 0;
                for (int l = 0; l < c.nc; l++) s += dd[k * c.nc + l] * B[l * ne + col];
                DB[k * ne + col] = s;
            }
        // upper triangle, mirrored: D is symmetric, so K is symmetric by construction
        for (int r = 0; r < ne; r++)
            for (int col = r; col < ne; col++) {
                double s = 0;
                for (int k = 0; k < c.nc; k++) s += B[k * ne + r] * DB[k * ne + col];
                K[r * ne + col] += coef * s;
            }
    }
    for (int r = 0; r < ne; r++)
        for (int col = 0; col < r; col++) K[r * ne + col] = K[col * ne + r];
    return 0;
}

// calculate_strain + update_stress at every IP (src/fem/element_solid.rs:190-224)
int elem_update(const ElemCtx& c, const double* X, int model, const Params& prm, const double* du /*nn*nd*/,
                double* sig, double* ivs, uint8_t* elastic, int* bad_ip) {
    IpGeo g;
    for (int p = 0; p < c.ngauss; p++) {
        int st = ip_geometry(c.kind, X, c.ksi + 3 * p, g);
        if (st) { if (bad_ip) *bad_ip = p; return st; }
        double eps[6] = {0, 0, 0, 0, 0, 0};
        if (c.nd == 2) {
            for (int m = 0; m < c.nn; m++) {
                double ux = du[2 * m], uy = du[2 * m + 1], gx = g.G[2 * m], gy = g.G[2 * m + 1];
                eps[0] += ux * gx;
                eps[1] += uy * gy;
                eps[3] += SQRT2 * ((ux * gy + uy * gx) / 2.0);
            }
            if (c.axisym) {  // src/base/calculate_strain.rs:36-48: out-of-plane strain u_r / r
                double r = 0.0;
                for (int m = 0; m < c.nn; m++) r += g.N[m] * X[2 * m];
                for (int m = 0; m < c.nn; m++) eps[2] += du[2 * m] * g.N[m] / r;
            }
        } else {
            for (int m = 0; m < c.nn; m++) {
                double ux = du[3 * m], uy = du[3 * m + 1], uz = du[3 * m + 2];
                double gx = g.G[3 * m], gy = g.G[3 * m + 1], gz = g.G[3 * m + 2];
                eps[0] += ux * gx;
                eps[1] += uy * gy;
                eps[2] += uz * gz;
                eps[3] += SQRT2 * ((ux * gy + uy * gx) / 2.0);
                eps[4] += SQRT2 * ((uy * gz + uz * gy) / 2.0);
                eps[5] += SQRT2 * ((ux * gz + uz * gx) / 2.0);
            }
        }
        st = model_update_stress(model, prm, c.nc, sig + p * c.nc, ivs + 2 * p, elastic + p, eps);
        if (st) { if (bad_ip) *bad_ip = p; return st; }
    }
    return 0;
}

void gather_X(const ElemCtx& c, const double* coords, const int64_t* conn, int64_t e, double* X) {
    for (int m = 0; m < c.nn; m++) {
        int64_t pt = conn[e * c.nn + m];
        for (int i = 0; i < c.nd; i++) X[m * c.nd + i] = coords[pt * c.nd + i];
    }
}

}  // namespace

// ------------------------------------------------------------------ general elastoplasticity
// Elastoplastic::update_stress (src/material/elastoplastic.rs:376-641) with the von Mises
// plasticity model (src/material/von_mises.rs:229-282), restated with dense Mandel matrices:
// D_e from elastic_modulus, D_ep = D_e - (D_e n)(n D_e)/N_p formed as a matrix
// (t4_ddot_t2_dyad_t2_ddot_t4), dsigma/dt = D_ep deps.  Intersection finding brackets the
// crossings of f(t) = sigma_d(sigma0 + t D_e deps) - z on the two monotone pieces of the convex f
// and refines them by bisection (the reference interpolates f with a Chebyshev series and finds
// its roots).
// The ODE is integrated with the Dormand-Prince 5(4) pair and the standard step controller (the
// reference uses DoPri8 from russell_ode, which is not available here).
// Returns 0, or 9 (df/dsigma singular), 10 (negative plastic numerator), 11 (ODE step limit),
// 12 (no crossing although the trial point is outside).  case: 0 AE, 1 AXB, 2 BE, 3 BXP, 4 BP.
namespace ep {

const double NUMERATOR_TOL = 1e-8;    // elastoplastic.rs:17
const double PSEUDO_TIME_TOL = 1e-7;  // elastoplastic.rs:23

double sigma_d_of(int nc, const double* v) {
    double m = (v[0] + v[1] + v[2]) / 3.0, q = 0;
    for (int i = 0; i < 3; i++) q += (v[i] - m) * (v[i] - m);
    for (int i = 3; i < nc; i++) q += v[i] * v[i];
    return std::sqrt(1.5 * q);
}

// f along the elastic path with z frozen
double f_path(int nc, const double* s0, const double* dse, double z, double t) {
    double v[6];
    for (int i = 0; i < nc; i++) v[i] = s0[i] + t * dse[i];
    return sigma_d_of(nc, v) - z;
}

// roots of f_path in [0, 1].  sigma_d is a norm of an affine function of t, so f is convex: it
// has at most one root on each side of its minimiser t_v.  Each monotone piece [0, t_v], [t_v, 1]
// is checked for a sign change and refined by bisection.
int roots(int nc, const double* s0, const double* dse, double z, double* r) {
    double m0 = (s0[0] + s0[1] + s0[2]) / 3.0, md = (dse[0] + dse[1] + dse[2]) / 3.0, sd = 0, dd = 0;
    for (int i = 0; i < nc; i++) {
        double a = (i < 3) ? s0[i] - m0 : s0[i], b = (i < 3) ? dse[i] - md : dse[i];
        sd += a * b;
        dd += b * b;
    }
    double tv = dd > 0 ? std::min(1.0, std::max(0.0, -sd / dd)) : 0.0;
    double cuts[3] = {0.0, tv, 1.0};
    int k = 0;
    for (int piece = 0; piece < 2; piece++) {
        double lo = cuts[piece], hi = cuts[piece + 1];
        if (!(hi > lo)) continue;
        double flo = f_path(nc, s0, dse, z, lo), fhi = f_path(nc, s0, dse, z, hi);
        bool change = (flo < 0.0) != (fhi < 0.0);
        if (piece == 0 && lo == 0.0 && flo == 0.0 && fhi < 0.0) {  // starts exactly on the surface
            r[k++] = 0.0;
            continue;
        }
        if (!change) continue;
        for (int it = 0; it < 200 && hi - lo > 1e-17; it++) {
            double mid = 0.5 * (lo + hi), fm = f_path(nc, s0, dse, z, mid);
            if ((fm < 0.0) == (flo < 0.0)) { lo = mid; flo = fm; } else hi = mid;
        }
        r[k++] = 0.5 * (lo + hi);
    }
    return k;
}

// dy/dt of y = [sigma, z] (elastoplastic.rs:159-205)
int rates(const Params& p, int nc, const double* De, const double* y, const double* deps, double* dy) {
    double m = (y[0] + y[1] + y[2]) / 3.0, s[6];
    for (int i = 0; i < nc; i++) s[i] = (i < 3) ? y[i] - m : y[i];
    double sd = sigma_d_of(nc, y);
    if (!(sd > 1e-10)) return 9;  // deriv1_invariant_sigma_d fails at sigma_d = 0
    double n[6], Den[6], nDe[6];
    for (int i = 0; i < nc; i++) n[i] = 1.5 * s[i] / sd;  // df/dsigma
    for (int i = 0; i < nc; i++) {
        Den[i] = 0; nDe[i] = 0;
        for (int j = 0; j < nc; j++) { Den[i] += De[i * nc + j] * n[j]; nDe[i] += n[j] * De[j * nc + i]; }
    }
    double mp = -(-1.0) * p.hh;  // M_p = -(df/dz) H_yf
    double nn = 0;
    for (int i = 0; i < nc; i++) nn += n[i] * Den[i];
    double np = mp + nn;
    double Dep[36];
    for (int i = 0; i < nc; i++)
        for (int j = 0; j < nc; j++) Dep[i * nc + j] = De[i * nc + j] - Den[i] * nDe[j] / np;
    double numerator = 0;
    for (int i = 0; i < nc; i++) numerator += nDe[i] * deps[i];
    for (int i = 0; i < nc; i++) {
        dy[i] = 0;
        for (int j = 0; j < nc; j++) dy[i] += Dep[i * nc + j] * deps[j];
    }
    if (numerator < -NUMERATOR_TOL) return 10;
    double lam_d = std::max(0.0, numerator) / np;
    dy[nc] = lam_d * p.hh;
    return 0;
}

int integrate(const Params& p, int nc, const double* De, double t0, double* y, const double* deps,
              double rtol, double atol, double h_ini, int max_steps, int* nstep) {
    static const double c_a[7][6] = {
        {0, 0, 0, 0, 0, 0},
        {1.0 / 5.0, 0, 0, 0, 0, 0},
        {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0},
        {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0},
        {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0},
        {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0},
        {35.0 / 384.0, 0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0}};
    static const double c_e[7] = {71.0 / 57600.0, 0, -71.0 / 16695.0, 71.0 / 1920.0, -17253.0 / 339200.0,
                                  22.0 / 525.0, -1.0 / 40.0};
    const int D = nc + 1;
    double k[7][7], yt[7], y5[7];
    double t = t0, h = std::min(h_ini, 1.0 - t0);
    int rc = rates(p, nc, De, y, deps, k[0]);
    if (rc) return rc;
    bool rejected = false;
    int steps = 0;
    while (t < 1.0) {
        if (steps >= max_steps) { *nstep = steps; return 11; }
        steps++;
        bool last = t + h >= 1.0;
        if (last) h = 1.0 - t;
        for (int st = 1; st < 7; st++) {
            for (int i = 0; i < D; i++) {
                double acc = 0;
                for (int j = 0; j < st; j++) acc += c_a[st][j] * k[j][i];
                yt[i] = y[i] + h * acc;
            }
            if (st == 6) for (int i = 0; i < D; i++) y5[i] = yt[i];
            rc = rates(p, nc, De, yt, deps, k[st]);
            if (rc) { *nstep = steps; return rc; }
        }
        double err = 0;
        for (int i = 0; i < D; i++) {
            double ei = 0;
            for (int j = 0; j < 7; j++) ei += c_e[j] * k[j][i];
            ei *= h;
            double sc = atol + rtol * std::max(std::fabs(y[i]), std::fabs(y5[i]));
            err += (ei / sc) * (ei / sc);
        }
        err = std::sqrt(err / D);
        double fac = err > 0 ? 0.9 * std::pow(err, -0.2) : 10.0;
        if (err <= 1.0) {
            t = last ? 1.0 : t + h;
            for (int i = 0; i < D; i++) { y[i] = y5[i]; k[0][i] = k[6][i]; }
            fac = std::min(rejected ? 1.0 : 10.0, std::max(0.2, fac));
            rejected = false;
        } else {
            fac = std::min(1.0, std::max(0.2, fac));
            rejected = true;
        }
        h *= fac;
    }
    *nstep = steps;
    return 0;
}

int update(const Params& p, int nc, double* sig, double* z, uint8_t* elastic, const double* deps, double rtol,
           double atol, double h_ini, int max_steps, int* cs, int* nstep) {
    double De[36], dse[6];
    elastic_modulus(p, nc, De);
    for (int i = 0; i < nc; i++) {
        dse[i] = 0;
        for (int j = 0; j < nc; j++) dse[i] += De[i * nc + j] * deps[j];
    }
    *nstep = 0;
    const double f0 = sigma_d_of(nc, sig) - *z;  // yield_function (von_mises.rs:236-240)
    double r[2], t_int = 0;
    int c;
    if (f0 < 0.0) {  // select_case: A (elastoplastic.rs:442-470)
        int nr = roots(nc, sig, dse, *z, r);
        if (nr == 0) {
            if (f_path(nc, sig, dse, *z, 1.0) > 0.0) return 12;
            c = 0;
        } else {
            t_int = r[0];
            c = (t_int <= PSEUDO_TIME_TOL) ? 4 : (t_int >= 1.0 - PSEUDO_TIME_TOL) ? 0 : 1;
        }
    } else {  // B (elastoplastic.rs:471-498); going_inside (:379-389)
        double sd = f0 + *z, indicator = 0;
        if (!(sd > 1e-10)) return 9;
        double m = (sig[0] + sig[1] + sig[2]) / 3.0, md = (dse[0] + dse[1] + dse[2]) / 3.0, nn = 0, dd = 0;
        for (int i = 0; i < nc; i++) {
            double ni = 1.5 * ((i < 3) ? sig[i] - m : sig[i]) / sd, di = (i < 3) ? dse[i] - md : dse[i];
            indicator += ni * dse[i];
            nn += ni * ni;
            dd += di * di;
        }
        // tangential loading (indicator zero up to rounding) does not count as going inside
        if (indicator < -1e-10 * std::sqrt(nn * dd)) {
            // the start (on or just outside the surface) gives the first crossing; a second one is
            // where the path leaves the surface again (elastoplastic.rs:420-427)
            int nr = roots(nc, sig, dse, *z, r);
            if (nr == 2) {
                t_int = r[1];
                c = (t_int <= PSEUDO_TIME_TOL) ? 4 : (t_int >= 1.0 - PSEUDO_TIME_TOL) ? 2 : 3;
            } else {
                if (f_path(nc, sig, dse, *z, 1.0) > 0.0) return 12;
                c = 2;
            }
        } else {
            c = 4;
        }
    }
    *cs = c;
    if (c == 0 || c == 2) {
        for (int i = 0; i < nc; i++) sig[i] += dse[i];
        *elastic = 1;
        return 0;
    }
    double y[7], t0 = (c == 4) ? 0.0 : t_int;
    for (int i = 0; i < nc; i++) y[i] = sig[i] + t0 * dse[i];
    y[nc] = *z;
    int rc = integrate(p, nc, De, t0, y, deps, rtol, atol, h_ini, max_steps, nstep);
    if (rc) return rc;
    for (int i = 0; i < nc; i++) sig[i] = y[i];
    *z = y[nc];
    *elastic = 0;
    return 0;
}

}  // namespace ep

extern "C" {

int orc_default_ngauss(int kind) { return default_ngauss(kind); }
int orc_kind_nnode(int kind) { return kind_nnode(kind); }

int orc_gauss(int kind, int ngauss, double* ksi, double* w) {
    if (ngauss <= 0) ngauss = default_ngauss(kind);
    return gauss_rule(kind, ngauss, ksi, w);
}

int orc_shape(int kind, const double* ksi, double* N, double* dN) {
    if (kind_nnode(kind) < 0) return -1;
    shape(kind, ksi, N, dN);
    return 0;
}

int orc_model_update_stress(int model, const double* prm, int ndim, double* sig, double* ivs, uint8_t* elastic,
                            const double* deps) {
    Params p{prm[0], prm[1], prm[2], prm[3]};
    return model_update_stress(model, p, 2 * ndim, sig, ivs, elastic, deps);
}

int orc_model_stiffness(int model, const double* prm, int ndim, const double* sig, const double* ivs,
                        uint8_t elastic, double* dd) {
    Params p{prm[0], prm[1], prm[2], prm[3]};
    return model_stiffness(model, p, 2 * ndim, sig, ivs, elastic, dd);
}

// Batched material call over n IPs, AoS state (sig n*nc, ivs n*2, elastic n); optional OpenMP.
int orc_model_update_and_stiffness_batch(int model, const double* prm, int ndim, int64_t n, double* sig, double* ivs,
                                         uint8_t* elastic, const double* deps, double* dd /*n*nc*nc or null*/,
                                         int nthreads) {
    Params p{prm[0], prm[1], prm[2], prm[3]};
    int nc = 2 * ndim;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : err)
#endif
    for (int64_t i = 0; i < n; i++) {
        int st = model_update_stress(model, p, nc, sig + i * nc, ivs + 2 * i, elastic + i, deps + i * nc);
        if (!st && dd) st = model_stiffness(model, p, nc, sig + i * nc, ivs + 2 * i, elastic[i], dd + i * nc * nc);
        if (st > err) err = st;
    }
    (void)nthreads;
    return err;
}

// The same batch with a hardening modulus per IP (hh[n]; prm[2] is ignored).
int orc_model_batch_hh(int model, const double* prm, int ndim, int64_t n, const double* hh, double* sig, double* ivs,
                       uint8_t* elastic, const double* deps, double* dd, int nthreads) {
    int nc = 2 * ndim;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(static) reduction(max : err)
#endif
    for (int64_t i = 0; i < n; i++) {
        Params p{prm[0], prm[1], hh[i], prm[3]};
        int st = model_update_stress(model, p, nc, sig + i * nc, ivs + 2 * i, elastic + i, deps + i * nc);
        if (!st && dd) st = model_stiffness(model, p, nc, sig + i * nc, ivs + 2 * i, elastic[i], dd + i * nc * nc);
        if (st > err) err = st;
    }
    (void)nthreads;
    return err;
}

int orc_elem_f_int(int kind, int ngauss, double thickness, const double* X, const double* sig, double* f) {
    ElemCtx c;
    if (!make_ctx(kind, ngauss, thickness, c)) return -1;
    return elem_f_int(c, X, sig, f);
}

int orc_elem_jacobian(int kind, int ngauss, double thickness, const double* X, int model, const double* prm,
                      const double* sig, const double* ivs, const uint8_t* elastic, double* K) {
    ElemCtx c;
    if (!make_ctx(kind, ngauss, thickness, c)) return -1;
    Params p{prm[0], prm[1], prm[2], prm[3]};
    return elem_jacobian(c, X, model, p, sig, ivs, elastic, K);
}

// ---- mesh level (Elements loops, src/fem/elements.rs:132-205) ----
// State arrays are per IP in cell-major order: ip_global = cell*ngauss + p.
// DOF numbering: eq = ndim*point + d (solid-only mesh, src/base/all_dofs.rs:87-116).

int orc_assemble_f_int(int kind, int ngauss, double thickness, int64_t npoint, const double* coords, int64_t ncell,
                       const int64_t* conn, const double* sig, double* ff /*npoint*nd, zeroed here*/) {
    ElemCtx c;
    if (!make_ctx(kind, ngauss, thickness, c)) return -1;
    int ne = c.nn * c.nd;
    for (int64_t i = 0; i < npoint * c.nd; i++) ff[i] = 0;
    double X[60], f[60];
    for (int64_t e = 0; e < ncell; e++) {
        gather_X(c, coords, conn, e, X);
        int st = elem_f_int(c, X, sig + e * c.ngauss * c.nc, f);
        if (st) return st;
        for (int l = 0; l < ne; l++) {
            int m = l / c.nd, i = l % c.nd;
            ff[conn[e * c.nn + m] * c.nd + i] += f[l];
        }
    }
    return 0;
}

// COO triplets with duplicates, element order, l-major / ll-minor (src/base/assembly.rs:120-135).
// rows/cols/vals hold ncell*ne*ne entries. sym_tol < 0 disables the symmetry check.
// nthreads > 1 runs elements in parallel (each writes its own slice, so the output is identical).
int orc_assemble_kk_coo(int kind, int ngauss, double thickness, const double* coords, int64_t ncell,
                        const int64_t* conn, int model, const double* prm, const double* sig, const double* ivs,
                        const uint8_t* elastic, double sym_tol, int64_t* rows, int64_t* cols, double* vals,
                        int nthreads, int64_t* bad_cell) {
    ElemCtx c;
    if (!make_ctx(kind, ngauss, thickness, c)) return -1;
    Params p{prm[0], prm[1], prm[2], prm[3]};
    int ne = c.nn * c.nd;
    int err = 0;
    int64_t bad = -1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
#endif
    {
        std::vector<double> K(ne * ne);
        double X[60];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int64_t e = 0; e < ncell; e++) {
            gather_X(c, coords, conn, e, X);
            int64_t ip0 = e * c.ngauss;
            int st = elem_jacobian(c, X, model, p, sig + ip0 * c.nc, ivs + ip0 * 2, elastic + ip0, K.data());
            if (!st && sym_tol >= 0) {
                for (int l = 0; l < ne && !st; l++)
                    for (int ll = l + 1; ll < ne; ll++)
                        if (std::fabs(K[l * ne + ll] - K[ll * ne + l]) > sym_tol) { st = 5; break; }
            }
            if (st) {
#ifdef _OPENMP
#pragma omp critical
#endif
                // the reference's loop stops at the first failing cell (src/fem/elements.rs:156-163)
                { if (err == 0 || e < bad) { err = st; bad = e; } }
                continue;
            }
            int64_t o = e * (int64_t)ne * ne;
            for (int l = 0; l < ne; l++) {
                int64_t g = conn[e * c.nn + l / c.nd] * c.nd + l % c.nd;
                for (int ll = 0; ll < ne; ll++) {
                    int64_t gg = conn[e * c.nn + ll / c.nd] * c.nd + ll % c.nd;
                    rows[o] = g; cols[o] = gg; vals[o] = K[l * ne + ll]; o++;
                }
            }
        }
    }
    (void)nthreads;
    if (bad_cell) *bad_cell = bad;
    return err;
}

// COO (with duplicates) -> CSR, summing duplicates in insertion order.
// Pass 1 (rowptr only): indptr must hold nrow+1; returns nnz.  Pass 2 fills indices/data.
int64_t orc_coo_to_csr(int64_t nrow, int64_t ntrip, const int64_t* rows, const int64_t* cols, const double* vals,
                       int64_t* indptr, int64_t* indices, double* data) {
    std::vector<int64_t> cnt(nrow + 1, 0);
    for (int64_t k = 0; k < ntrip; k++) cnt[rows[k] + 1]++;
    for (int64_t r = 0; r < nrow; r++) cnt[r + 1] += cnt[r];
    std::vector<int64_t> order(ntrip);
    {
        std::vector<int64_t> pos(cnt.begin(), cnt.end() - 1);
        for (int64_t k = 0; k < ntrip; k++) order[pos[rows[k]]++] = k;
    }
    int64_t nnz = 0;
    std::vector<int64_t> rowptr(nrow + 1, 0);
    std::vector<int64_t> tmp;
    for (int64_t r = 0; r < nrow; r++) {
        int64_t a = cnt[r], b = cnt[r + 1];
        tmp.assign(order.begin() + a, order.begin() + b);
        std::stable_sort(tmp.begin(), tmp.end(), [&](int64_t x, int64_t y) { return cols[x] < cols[y]; });
        int64_t prev = -1;
        for (int64_t k : tmp) {
            if (cols[k] != prev) {
                if (indices) { indices[nnz] = cols[k]; data[nnz] = vals[k]; }
                nnz++;
                prev = cols[k];
            } else if (indices) {
                data[nnz - 1] += vals[k];
            }
        }
        rowptr[r + 1] = nnz;
    }
    if (indptr) std::memcpy(indptr, rowptr.data(), (nrow + 1) * sizeof(int64_t));
    return nnz;
}

// update_secondary_values over all cells; ddu is the global (step) displacement increment.
int orc_update_secondary(int kind, int ngauss, double thickness, const double* coords, int64_t ncell,
                         const int64_t* conn, int model, const double* prm, const double* ddu, double* sig,
                         double* ivs, uint8_t* elastic, int nthreads, int64_t* bad_cell, int* bad_ip) {
    ElemCtx c;
    if (!make_ctx(kind, ngauss, thickness, c)) return -1;
    Params p{prm[0], prm[1], prm[2], prm[3]};
    int err = 0;
    int64_t bc = -1;
    int bi = -1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 64)
#endif
    for (int64_t e = 0; e < ncell; e++) {
        double X[60], du[60];
        gather_X(c, coords, conn, e, X);
        for (int m = 0; m < c.nn; m++)
            for (int i = 0; i < c.nd; i++) du[m * c.nd + i] = ddu[conn[e * c.nn + m] * c.nd + i];
        int64_t ip0 = e * c.ngauss;
        int ip = -1;
        int st = elem_update(c, X, model, p, du, sig + ip0 * c.nc, ivs + ip0 * 2, elastic + ip0, &ip);
        if (st) {
#ifdef _OPENMP
#pragma omp critical
#endif
            // the first failing cell in the reference's loop order (src/fem/elements.rs:176-181)
            { if (err == 0 || e < bc) { err = st; bc = e; bi = ip; } }
        }
    }
    (void)nthreads;
    if (bad_cell) *bad_cell = bc;
    if (bad_ip) *bad_ip = bi;
    return err;
}

// General elastoplastic update over n IPs (AoS: sig n*nc, z n, elastic n, deps n*nc);
// settings = [rtol, atol, h_ini]; cases/steps per IP.  Returns the first error code (its IP in *bad).
int orc_ep_update_batch(const double* prm, int ndim, int64_t n, double* sig, double* z, uint8_t* elastic,
                        const double* deps, const double* settings, int max_steps, int32_t* cases, int32_t* steps,
                        int64_t* bad) {
    Params p{prm[0], prm[1], prm[2], prm[3]};
    int nc = 2 * ndim, err = 0;
    for (int64_t i = 0; i < n; i++) {
        double s[6], zi = z[i];
        uint8_t el = elastic[i];
        for (int c = 0; c < nc; c++) s[c] = sig[i * nc + c];
        int cs = -1, ns = 0;
        int st = ep::update(p, nc, s, &zi, &el, deps + i * nc, settings[0], settings[1], settings[2], max_steps,
                            &cs, &ns);
        if (st) {
            if (!err) { err = st; if (bad) *bad = i; }
            cs = -1;
        } else {
            for (int c = 0; c < nc; c++) sig[i * nc + c] = s[c];
            z[i] = zi;
            elastic[i] = el;
        }
        cases[i] = cs;
        steps[i] = ns;
    }
    return err;
}

int orc_max_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
