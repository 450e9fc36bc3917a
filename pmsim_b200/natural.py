"""Natural boundary conditions: distributed loads on cell sides and concentrated point loads.

Mirrors ``Natural`` / ``BcDistributed`` / ``BcConcentrated`` of the reference
(``src/base/natural.rs``, ``src/fem/bc_distributed.rs``, ``src/fem/bc_concentrated.rs``): the
external force vector is F_ext(t) = sum over loads of value * f(t) * (consistent nodal forces).
A distributed load on a side (edge in 2D, face in 3D) gives f_m = int N_m q dA with q = qn * n
(outward unit normal, ``Nbc::Qn``) or a fixed direction (``Nbc::Qx/Qy/Qz``), integrated with a
Gauss rule that is exact for the side's polynomial degree.  Sides are found as in gemlab's
``Features::search_edges/search_faces``: every node of the side lies on the locus and satisfies
the optional filter.
"""
from __future__ import annotations

import numpy as np

from . import mesh as M

# local sides of each kind: corners in order, then the side's mid nodes (quadratic kinds);
# a side is a line (2D) or a tri/quad face (3D)
SIDES = {
    M.TRI3: [[0, 1], [1, 2], [2, 0]],
    M.TRI6: [[0, 1, 3], [1, 2, 4], [2, 0, 5]],
    M.QUA4: [[0, 1], [1, 2], [2, 3], [3, 0]],
    M.QUA8: [[0, 1, 4], [1, 2, 5], [2, 3, 6], [3, 0, 7]],
    M.QUA9: [[0, 1, 4], [1, 2, 5], [2, 3, 6], [3, 0, 7]],
    M.TET4: [[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]],
    M.TET10: [[0, 2, 1, 6, 5, 4], [0, 1, 3, 4, 8, 7], [0, 3, 2, 7, 9, 6], [1, 2, 3, 5, 9, 8]],
    M.HEX8: [[0, 4, 7, 3], [1, 2, 6, 5], [0, 1, 5, 4], [2, 3, 7, 6], [0, 3, 2, 1], [4, 5, 6, 7]],
    M.HEX20: [[0, 4, 7, 3, 16, 15, 19, 11], [1, 2, 6, 5, 9, 18, 13, 17], [0, 1, 5, 4, 8, 17, 12, 16],
              [2, 3, 7, 6, 10, 19, 14, 18], [0, 3, 2, 1, 11, 10, 9, 8], [4, 5, 6, 7, 12, 13, 14, 15]],
}

_G3 = (np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)]), np.array([5.0, 8.0, 5.0]) / 9.0)


def _line_shape(n, s):
    """Lin2 / Lin3 (corners at s = -1, +1, mid at 0) on [-1, 1]."""
    if n == 2:
        return np.array([(1 - s) / 2, (1 + s) / 2]), np.array([[-0.5], [0.5]])
    return (np.array([s * (s - 1) / 2, s * (s + 1) / 2, 1 - s * s]),
            np.array([[s - 0.5], [s + 0.5], [-2 * s]]))


def _face_shape(n, r, s):
    """Quad faces (4 or 8 nodes: corners CCW, then mid-edges) on [-1,1]^2; tri faces (3 or 6 nodes)."""
    if n in (4, 8):
        xi = [(-1, -1), (1, -1), (1, 1), (-1, 1), (0, -1), (1, 0), (0, 1), (-1, 0)]
        N = np.zeros(n)
        dN = np.zeros((n, 2))
        for m in range(n):
            a, b = xi[m]
            if n == 4:
                N[m] = (1 + a * r) * (1 + b * s) / 4
                dN[m] = [a * (1 + b * s) / 4, b * (1 + a * r) / 4]
            elif m < 4:
                N[m] = (1 + a * r) * (1 + b * s) * (a * r + b * s - 1) / 4
                dN[m] = [a * (1 + b * s) * (2 * a * r + b * s) / 4, b * (1 + a * r) * (a * r + 2 * b * s) / 4]
            elif a == 0:
                N[m] = (1 - r * r) * (1 + b * s) / 2
                dN[m] = [-r * (1 + b * s), b * (1 - r * r) / 2]
            else:
                N[m] = (1 + a * r) * (1 - s * s) / 2
                dN[m] = [a * (1 - s * s) / 2, -s * (1 + a * r)]
        return N, dN
    L = np.array([1 - r - s, r, s])
    dL = np.array([[-1, -1], [1, 0], [0, 1]], dtype=float)
    if n == 3:
        return L, dL
    N = np.zeros(6)
    dN = np.zeros((6, 2))
    for m in range(3):
        N[m] = L[m] * (2 * L[m] - 1)
        dN[m] = (4 * L[m] - 1) * dL[m]
    for e, (i, j) in enumerate([(0, 1), (1, 2), (2, 0)]):
        N[3 + e] = 4 * L[i] * L[j]
        dN[3 + e] = 4 * (dL[i] * L[j] + L[i] * dL[j])
    return N, dN


def _face_rule(n):
    if n in (4, 8):
        x, w = _G3
        return [(a, b, wa * wb) for b, wb in zip(x, w) for a, wa in zip(x, w)]
    # 6-point rule on the reference triangle (degree 4)
    a, b = 0.445948490915965, 0.091576213509771
    wa, wb = 0.223381589678011 / 2, 0.109951743655322 / 2
    return [(a, a, wa), (1 - 2 * a, a, wa), (a, 1 - 2 * a, wa), (b, b, wb), (1 - 2 * b, b, wb), (b, 1 - 2 * b, wb)]


def find_sides(mesh: M.Mesh, on_locus, filt=None):
    """(cell, local side) of every side whose nodes all satisfy on_locus(x) and filt(x)."""
    out = []
    seen = set()
    for c in range(mesh.ncell):
        for k, side in enumerate(SIDES[mesh.kind]):
            pts = mesh.cells[c][side]
            X = mesh.coords[pts]
            if all(on_locus(x) for x in X) and (filt is None or all(filt(x) for x in X)):
                key = tuple(sorted(pts[: (2 if mesh.ndim == 2 else (4 if len(side) in (4, 8) else 3))]))
                if key not in seen:
                    seen.add(key)
                    out.append((c, k))
    return out


def side_forces(mesh: M.Mesh, sides, component=None, axisymmetric=False, thickness=1.0):
    """Consistent nodal forces of a unit load on the sides: component=None -> unit outward normal
    pressure (qn = 1), else unit traction along axis `component`.  In the axisymmetric idealization
    (2D, x = radius) the side integral carries the radius, f_m = int N_m q r dl (per radian), as the
    element integrals do; otherwise a 2D side integral carries the thickness (args.alpha in
    src/fem/bc_distributed.rs:139-165)."""
    nd = mesh.ndim
    f = np.zeros(mesh.ndof)
    for c, k in sides:
        local = SIDES[mesh.kind][k]
        pts = mesh.cells[c][local]
        X = mesh.coords[pts]
        centroid = mesh.coords[mesh.cells[c]].mean(0)
        n = len(local)
        if nd == 2:
            x, w = _G3
            for s, ws in zip(x, w):
                N, dN = _line_shape(n, s)
                t = X.T @ dN[:, 0]  # dx/ds
                normal = np.array([t[1], -t[0]])  # |normal| = |dx/ds| (the length factor)
                if np.dot(N @ X - centroid, normal) < 0:
                    normal = -normal
                q = normal if component is None else np.eye(2)[component] * np.linalg.norm(t)
                if axisymmetric:
                    q = q * (N @ X[:, 0])
                elif thickness != 1.0:
                    q = q * thickness
                for m in range(n):
                    f[nd * pts[m]: nd * pts[m] + nd] += ws * N[m] * q
        else:
            for r, s, ws in _face_rule(n):
                N, dN = _face_shape(n, r, s)
                tr, ts = X.T @ dN[:, 0], X.T @ dN[:, 1]
                normal = np.cross(tr, ts)  # |normal| = area factor
                if np.dot(N @ X - centroid, normal) < 0:
                    normal = -normal
                q = normal if component is None else np.eye(3)[component] * np.linalg.norm(normal)
                for m in range(n):
                    f[nd * pts[m]: nd * pts[m] + nd] += ws * N[m] * q
    return f


class Natural:
    """Loads as (unit force vector, value, f(t) or None); ff_ext(t) = sum value * f(t) * unit."""

    def __init__(self, mesh: M.Mesh, axisymmetric=False, thickness=1.0):
        self.mesh = mesh
        self.axisymmetric = bool(axisymmetric)
        self.thickness = float(thickness)
        if self.axisymmetric and mesh.ndim != 2:
            raise ValueError("the axisymmetric idealization is two-dimensional")
        self.items = []

    def sides(self, sides, value, fn=None, component=None):
        self.items.append((side_forces(self.mesh, sides, component, self.axisymmetric, self.thickness), float(value),
                           fn))
        return self

    def points(self, point_ids, dof, value, fn=None):
        u = np.zeros(self.mesh.ndof)
        for p in point_ids:
            u[self.mesh.ndim * int(p) + dof] += 1.0
        self.items.append((u, float(value), fn))
        return self

    def ff_ext(self, t):
        f = np.zeros(self.mesh.ndof)
        for unit, v, fn in self.items:
            f += (v * fn(t) if fn is not None else v) * unit
        return f
