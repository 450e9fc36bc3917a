// pms_shapes.cpp -- see pms_shapes.h.
#include "pms_shapes.h"

#include <cmath>

namespace pms {

namespace {
const int NNODE[9] = {3, 6, 4, 8, 9, 4, 10, 8, 20};
const int NDIM[9] = {2, 2, 2, 2, 2, 3, 3, 3, 3};
const int NGAUSS_DEFAULT[9] = {3, 3, 4, 9, 9, 4, 4, 8, 27};

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

int kind_nnode(int kind) { return (kind >= 0 && kind < 9) ? NNODE[kind] : -1; }
int kind_ndim(int kind) { return (kind >= 0 && kind < 9) ? NDIM[kind] : -1; }
int kind_default_ngauss(int kind) { return (kind >= 0 && kind < 9) ? NGAUSS_DEFAULT[kind] : -1; }

int integration_rule(int kind, int ngauss, std::vector<double>& ksi, std::vector<double>& w) {
    if (kind < 0 || kind > 8) return -1;
    if (ngauss <= 0) ngauss = NGAUSS_DEFAULT[kind];
    int nd = NDIM[kind];
    ksi.assign(3 * ngauss, 0.0);
    w.assign(ngauss, 0.0);
    const bool simplex = (kind == 0 || kind == 1 || kind == 5 || kind == 6);
    if (!simplex) {
        int n1 = (int)std::lround(std::pow((double)ngauss, 1.0 / nd));
        int tot = 1;
        for (int d = 0; d < nd; d++) tot *= n1;
        if (n1 < 1 || n1 > 3 || tot != ngauss) return -1;
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
    if (nd == 2) {
        if (ngauss == 1) {
            ksi[0] = ksi[1] = 1.0 / 3.0;
            w[0] = 0.5;
            return 1;
        }
        if (ngauss == 3) {
            const double lo = 1.0 / 6.0, hi = 2.0 / 3.0;
            const double pts[3][2] = {{lo, lo}, {hi, lo}, {lo, hi}};
            for (int p = 0; p < 3; p++) {
                ksi[3 * p] = pts[p][0];
                ksi[3 * p + 1] = pts[p][1];
                w[p] = 1.0 / 6.0;
            }
            return 3;
        }
        return -1;
    }
    if (ngauss == 1) {
        ksi[0] = ksi[1] = ksi[2] = 0.25;
        w[0] = 1.0 / 6.0;
        return 1;
    }
    if (ngauss == 4) {
        const double hi = (5.0 + 3.0 * std::sqrt(5.0)) / 20.0, lo = (5.0 - std::sqrt(5.0)) / 20.0;
        for (int p = 0; p < 4; p++) {
            for (int d = 0; d < 3; d++) ksi[3 * p + d] = (p > 0 && d == p - 1) ? hi : lo;
            w[p] = 1.0 / 24.0;
        }
        return 4;
    }
    return -1;
}

int integration_rule_into(int kind, int ngauss, double* ksi, double* w) {
    if (kind < 0 || kind > 8) return -1;
    if (ngauss <= 0) ngauss = NGAUSS_DEFAULT[kind];
    if (ngauss > 27) return -1;
    const int nd = NDIM[kind];
    for (int i = 0; i < 3 * ngauss; i++) ksi[i] = 0.0;
    const bool simplex = (kind == 0 || kind == 1 || kind == 5 || kind == 6);
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
    return -1;
}

void shape_eval(int kind, const double* k, double* N, double* dN) {
    const double r = k[0], s = k[1], t = k[2];
    switch (kind) {
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
