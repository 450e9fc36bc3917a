// pms_shapes.cpp -- see pms_shapes.h.
#include "pms_shapes.h"

#include <cmath>

namespace pms {

namespace {
constexpr int NKIND = 11;
const int NNODE[NKIND] = {3, 6, 4, 8, 9, 4, 10, 8, 20, 10, 15};
const int NDIM[NKIND] = {2, 2, 2, 2, 2, 3, 3, 3, 3, 2, 2};
// Tri10 / Tri15: the lowest symmetric rule that integrates the stiffness of a straight-sided cell
// exactly (degree 4 and 6)
const int NGAUSS_DEFAULT[NKIND] = {3, 3, 4, 9, 9, 4, 4, 8, 27, 6, 12};
bool simplex_kind(int kind) { return kind == 0 || kind == 1 || kind == 5 || kind == 6 || kind == 9 || kind == 10; }

// Barycentric positions (i, j, k)/n of the nodes of the cubic (n = 3) and quartic (n = 4) triangles:
// corners; for n = 4 the mid-edge nodes of edges 0-1, 1-2, 2-0; then per edge the node nearer its
// first corner and the one nearer its second; then the interior nodes (the Tri15 order of the
// reference's meshes, src/base/sample_meshes.rs:305-362).
const int TRI10_POS[10][3] = {{3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {2, 1, 0}, {1, 2, 0},
                              {0, 2, 1}, {0, 1, 2}, {1, 0, 2}, {2, 0, 1}, {1, 1, 1}};
const int TRI15_POS[15][3] = {{4, 0, 0}, {0, 4, 0}, {0, 0, 4}, {2, 2, 0}, {0, 2, 2}, {2, 0, 2}, {3, 1, 0}, {1, 3, 0},
                              {0, 3, 1}, {0, 1, 3}, {1, 0, 3}, {3, 0, 1}, {2, 1, 1}, {1, 2, 1}, {1, 1, 2}};

// Silvester's factor of a complete Lagrange triangle of order n: P_a(L) = prod_{q<a} (n L - q)/(q + 1)
// and its derivative in L (Zienkiewicz & Taylor, Vol. 1, sec. 6.6).
void silvester_factor(int n, int a, double L, double& P, double& dP) {
    P = 1.0;
    dP = 0.0;
    for (int q = 0; q < a; q++) {
        const double f = (n * L - q) / (q + 1);
        dP = dP * f + P * n / (q + 1);
        P *= f;
    }
}

// Symmetric triangle rules of Dunavant (1985, Int. J. Numer. Meth. Eng. 21:1129-1148) on the
// reference triangle (area 1/2): orbit type 1 = centroid, 3 = (a, a, 1 - 2a) and its rotations,
// 6 = (a, b, 1 - a - b) and its permutations; weights given for unit area.
int triangle_rule(int ngauss, double* ksi, double* w) {
    struct Orbit { int type; double w, a, b; };
    Orbit orb[3];
    int norb = 0;
    const double r15 = std::sqrt(15.0);
    switch (ngauss) {
    case 6:  // degree 4
        orb[0] = {3, 0.223381589678011, 0.445948490915965, 0.0};
        orb[1] = {3, 0.109951743655322, 0.091576213509771, 0.0};
        norb = 2;
        break;
    case 7:  // degree 5 (closed form)
        orb[0] = {1, 0.225, 1.0 / 3.0, 0.0};
        orb[1] = {3, (155.0 + r15) / 1200.0, (6.0 + r15) / 21.0, 0.0};
        orb[2] = {3, (155.0 - r15) / 1200.0, (6.0 - r15) / 21.0, 0.0};
        norb = 3;
        break;
    case 12:  // degree 6
        orb[0] = {3, 0.116786275726379, 0.249286745170910, 0.0};
        orb[1] = {3, 0.050844906370207, 0.063089014491502, 0.0};
        orb[2] = {6, 0.082851075618374, 0.053145049844817, 0.310352451033784};
        norb = 3;
        break;
    default:
        return -1;
    }
    int p = 0;
    for (int o = 0; o < norb; o++) {
        const double a = orb[o].a, b = orb[o].b;
        double pts[6][2];
        int n = 1;
        pts[0][0] = pts[0][1] = a;
        if (orb[o].type == 3) {
            const double c = 1.0 - 2.0 * a;
            pts[1][0] = c; pts[1][1] = a;
            pts[2][0] = a; pts[2][1] = c;
            n = 3;
        } else if (orb[o].type == 6) {
            const double c = 1.0 - a - b;
            const double q[6][2] = {{a, b}, {b, a}, {b, c}, {c, b}, {c, a}, {a, c}};
            for (int i = 0; i < 6; i++) { pts[i][0] = q[i][0]; pts[i][1] = q[i][1]; }
            n = 6;
        }
        for (int i = 0; i < n; i++, p++) {
            ksi[3 * p] = pts[i][0];
            ksi[3 * p + 1] = pts[i][1];
            ksi[3 * p + 2] = 0.0;
            w[p] = 0.5 * orb[o].w;
        }
    }
    return p;
}

// natural coordinates of the nodes of the hypercube kinds (corners first)
const double QUA_NODES[9][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}, {0, -1}, {1, 0}, {0, 1}, {-1, 0}, {0, 0}};
const double HEX_NODES[20][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
    {0, -1, -1},  {1, 0, -1},  {0, 1, -1}, {-1, 0, -1}, {0, -1, 1},  {1, 0, 1},  {0, 1, 1}, {-1, 0, 1},
    {-1, -1, 0},  {1, -1, 0},  {1, 1, 0},  {-1, 1, 0}};

// 1D quadratic Lagrange polynomials on {-1, 0, 1}, indexed by the node coordinate
inline double lag2(double c, double x) { return c < 0 ? 0.5 * x * (x - 1) : (c > 0 ? 0.5 * x * (x + 1) : 1 - x * x); }
inline double dlag2(double c, double x) { return c < 0 ? x - 0.5 : (c > 0 ? x + 0.5 : -2 * x); }

void gauss_legendre(int n, double* x, double* w) {
    if (n == 1) {
        x[0] = 0;
        w[0] = 2;
    } else if (n == 2) {
        x[1] = 1.0 / std::sqrt(3.0);
        x[0] = -x[1];
        w[0] = w[1] = 1;
    } else {
        x[2] = std::sqrt(0.6);
        x[1] = 0;
        x[0] = -x[2];
        w[0] = w[2] = 5.0 / 9.0;
        w[1] = 8.0 / 9.0;
    }
}
}  // namespace

int kind_nnode(int kind) { return (kind >= 0 && kind < NKIND) ? NNODE[kind] : -1; }
int kind_ndim(int kind) { return (kind >= 0 && kind < NKIND) ? NDIM[kind] : -1; }
int kind_default_ngauss(int kind) { return (kind >= 0 && kind < NKIND) ? NGAUSS_DEFAULT[kind] : -1; }

int integration_rule(int kind, int ngauss, std::vector<double>& ksi, std::vector<double>& w) {
    double k[3 * 27], ww[27];
    const int n = integration_rule_into(kind, ngauss, k, ww);
    if (n <= 0) return -1;
    ksi.assign(k, k + 3 * n);
    w.assign(ww, ww + n);
    return n;
}

int integration_rule_into(int kind, int ngauss, double* ksi, double* w) {
    if (kind < 0 || kind >= NKIND) return -1;
    if (ngauss <= 0) ngauss = NGAUSS_DEFAULT[kind];
    if (ngauss > 27) return -1;
    const int nd = NDIM[kind];
    for (int i = 0; i < 3 * ngauss; i++) ksi[i] = 0.0;
    const bool simplex = simplex_kind(kind);
    if (!simplex) {
        int n1 = 0;
        for (int c = 1; c <= 3; c++)
            if ((nd == 2 ? c * c : c * c * c) == ngauss) n1 = c;
        if (n1 == 0) return -1;
        double x[3], ww[3];
        gauss_legendre(n1, x, ww);
        for (int p = 0; p < ngauss; p++) {
            int i = p % n1, j = (p / n1) % n1, k = p / (n1 * n1);
            ksi[3 * p] = x[i];
            ksi[3 * p + 1] = x[j];
            ksi[3 * p + 2] = nd == 3 ? x[k] : 0.0;
            w[p] = ww[i] * ww[j] * (nd == 3 ? ww[k] : 1.0);
        }
        return ngauss;
    }
    if (ngauss == 1) {
        ksi[0] = ksi[1] = (nd == 2) ? 1.0 / 3.0 : 0.25;
        if (nd == 3) ksi[2] = 0.25;
        w[0] = (nd == 2) ? 0.5 : 1.0 / 6.0;
        return 1;
    }
    if (nd == 2 && ngauss == 3) {
        const double lo = 1.0 / 6.0, hi = 2.0 / 3.0;
        const double pts[3][2] = {{lo, lo}, {hi, lo}, {lo, hi}};
        for (int p = 0; p < 3; p++) {
            ksi[3 * p] = pts[p][0];
            ksi[3 * p + 1] = pts[p][1];
            w[p] = 1.0 / 6.0;
        }
        return 3;
    }
    if (nd == 3 && ngauss == 4) {
        const double hi = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, lo = (5.0 - std::sqrt(5.0)) / 20.0;
        for (int p = 0; p < 4; p++) {
            for (int d = 0; d < 3; d++) ksi[3 * p + d] = (p > 0 && d == p - 1) ? hi : lo;
            w[p] = 1.0 / 24.0;
        }
        return 4;
    }
    if (nd == 2) return triangle_rule(ngauss, ksi, w);
    return -1;
}

void shape_eval(int kind, const double* k, double* N, double* dN) {
    const double r = k[0], s = k[1], t = k[2];
    switch (kind) {
    case 9:    // Tri10: complete cubic triangle
    case 10: {  // Tri15: complete quartic triangle
        const int n = kind == 9 ? 3 : 4, nn = kind == 9 ? 10 : 15;
        const int(*pos)[3] = kind == 9 ? TRI10_POS : TRI15_POS;
        const double L0 = 1.0 - r - s;  // area coordinates (L0, L1, L2) = (1 - r - s, r, s)
        for (int m = 0; m < nn; m++) {
            double P0, d0, P1, d1, P2, d2;
            silvester_factor(n, pos[m][0], L0, P0, d0);
            silvester_factor(n, pos[m][1], r, P1, d1);
            silvester_factor(n, pos[m][2], s, P2, d2);
            N[m] = P0 * P1 * P2;
            dN[2 * m] = P0 * d1 * P2 - d0 * P1 * P2;
            dN[2 * m + 1] = P0 * P1 * d2 - d0 * P1 * P2;
        }
        break;
    }
    case 2:  // Qua4: bilinear
        for (int m = 0; m < 4; m++) {
            double a = QUA_NODES[m][0], b = QUA_NODES[m][1];
            N[m] = 0.25 * (1 + a * r) * (1 + b * s);
            dN[2 * m] = 0.25 * a * (1 + b * s);
            dN[2 * m + 1] = 0.25 * b * (1 + a * r);
        }
        break;
    case 3:  // Qua8: serendipity
        for (int m = 0; m < 8; m++) {
            double a = QUA_NODES[m][0], b = QUA_NODES[m][1];
            if (m < 4) {
                N[m] = 0.25 * (1 + a * r) * (1 + b * s) * (a * r + b * s - 1);
                dN[2 * m] = 0.25 * a * (1 + b * s) * (2 * a * r + b * s);
                dN[2 * m + 1] = 0.25 * b * (1 + a * r) * (a * r + 2 * b * s);
            } else if (a == 0) {
                N[m] = 0.5 * (1 - r * r) * (1 + b * s);
                dN[2 * m] = -r * (1 + b * s);
                dN[2 * m + 1] = 0.5 * b * (1 - r * r);
            } else {
                N[m] = 0.5 * (1 + a * r) * (1 - s * s);
                dN[2 * m] = 0.5 * a * (1 - s * s);
                dN[2 * m + 1] = -s * (1 + a * r);
            }
        }
        break;
    case 4:  // Qua9: tensor-product quadratic Lagrange
        for (int m = 0; m < 9; m++) {
            double a = QUA_NODES[m][0], b = QUA_NODES[m][1];
            N[m] = lag2(a, r) * lag2(b, s);
            dN[2 * m] = dlag2(a, r) * lag2(b, s);
            dN[2 * m + 1] = lag2(a, r) * dlag2(b, s);
        }
        break;
    case 7:  // Hex8: trilinear
        for (int m = 0; m < 8; m++) {
            double a = HEX_NODES[m][0], b = HEX_NODES[m][1], c = HEX_NODES[m][2];
            double fa = 1 + a * r, fb = 1 + b * s, fc = 1 + c * t;
            N[m] = 0.125 * fa * fb * fc;
            dN[3 * m] = 0.125 * a * fb * fc;
            dN[3 * m + 1] = 0.125 * b * fa * fc;
            dN[3 * m + 2] = 0.125 * c * fa * fb;
        }
        break;
    case 8:  // Hex20: serendipity
        for (int m = 0; m < 20; m++) {
            double a = HEX_NODES[m][0], b = HEX_NODES[m][1], c = HEX_NODES[m][2];
            double fa = 1 + a * r, fb = 1 + b * s, fc = 1 + c * t;
            if (m < 8) {
                double q = a * r + b * s + c * t - 2;
                N[m] = 0.125 * fa * fb * fc * q;
                dN[3 * m] = 0.125 * a * fb * fc * (q + fa);
                dN[3 * m + 1] = 0.125 * b * fa * fc * (q + fb);
                dN[3 * m + 2] = 0.125 * c * fa * fb * (q + fc);
            } else if (a == 0) {
                N[m] = 0.25 * (1 - r * r) * fb * fc;
                dN[3 * m] = -0.5 * r * fb * fc;
                dN[3 * m + 1] = 0.25 * (1 - r * r) * b * fc;
                dN[3 * m + 2] = 0.25 * (1 - r * r) * fb * c;
            } else if (b == 0) {
                N[m] = 0.25 * fa * (1 - s * s) * fc;
                dN[3 * m] = 0.25 * a * (1 - s * s) * fc;
                dN[3 * m + 1] = -0.5 * s * fa * fc;
                dN[3 * m + 2] = 0.25 * fa * (1 - s * s) * c;
            } else {
                N[m] = 0.25 * fa * fb * (1 - t * t);
                dN[3 * m] = 0.25 * a * fb * (1 - t * t);
                dN[3 * m + 1] = 0.25 * fa * b * (1 - t * t);
                dN[3 * m + 2] = -0.5 * t * fa * fb;
            }
        }
        break;
    default: {  // simplices in area/volume coordinates L0 = 1 - sum(ksi), Li = ksi_{i-1}
        const int nd = NDIM[kind];
        const int nv = nd + 1;
        double L[4] = {1 - r - s - (nd == 3 ? t : 0.0), r, s, t};
        double dL[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
        const bool quadratic = (kind == 1 || kind == 6);
        for (int m = 0; m < nv; m++) {
            N[m] = quadratic ? L[m] * (2 * L[m] - 1) : L[m];
            for (int j = 0; j < nd; j++) dN[nd * m + j] = (quadratic ? (4 * L[m] - 1) : 1.0) * dL[m][j];
        }
        if (quadratic) {
            // mid-edge nodes: Tri6 0-1, 1-2, 2-0; Tet10 0-1, 1-2, 2-0, 0-3, 1-3, 2-3
            const int edges[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 3}, {1, 3}, {2, 3}};
            int ne = (nd == 2) ? 3 : 6;
            for (int e = 0; e < ne; e++) {
                int i = edges[e][0], j = edges[e][1], m = nv + e;
                N[m] = 4 * L[i] * L[j];
                for (int d = 0; d < nd; d++) dN[nd * m + d] = 4 * (dL[i][d] * L[j] + L[i] * dL[j][d]);
            }
        }
    } break;
    }
}

}  // namespace pms
