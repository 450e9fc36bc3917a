// pms_shapes.h -- shape-function gradients and integration rules, tabulated once per element
// kind on the host and staged into shared memory by the element kernels.
//
// Replaces gemlab's Scratchpad/Gauss (called from src/fem/element_solid.rs:62,134,173,179 and
// src/base/calculate_strain.rs:27 of the reference).  Families (Zienkiewicz & Taylor, vol. 1):
//   * multilinear Qua4/Hex8, serendipity Qua8/Hex20, biquadratic Lagrange Qua9,
//   * linear/quadratic simplex Tri3/Tri6/Tet4/Tet10 in area/volume coordinates, and the complete
//     cubic/quartic triangles Tri10/Tri15 (Silvester's formula);
// Gauss-Legendre tensor rules (x fastest, then y, then z), interior simplex rules, and Dunavant's
// symmetric triangle rules of 6, 7 and 12 points.
// Node orders: corners (counter-clockwise / bottom then top), then mid-edges in the order
// 0-1, 1-2, 2-3, 3-0 (Qua8/Qua9, center last), and for Hex20 bottom, top, vertical mid-edges.
#pragma once
#include <vector>

namespace pms {

int kind_nnode(int kind);
int kind_ndim(int kind);
int kind_default_ngauss(int kind);

// Fills ksi[ngauss*3], w[ngauss].  Returns the number of points or -1.
int integration_rule(int kind, int ngauss, std::vector<double>& ksi, std::vector<double>& w);

// Same rules written into caller-provided arrays ksi[3*27], w[27] (no heap use).
int integration_rule_into(int kind, int ngauss, double* ksi, double* w);

// N[nn], dN[nn*nd] (dN_m/dksi_j) at one natural point.
void shape_eval(int kind, const double* ksi, double* N, double* dN);

}  // namespace pms
