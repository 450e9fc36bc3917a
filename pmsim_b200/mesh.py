"""Meshes for the solid hot path: a plain container plus structured generators.

The container mirrors the pieces of gemlab's ``Mesh`` that the element boundary reads
(``ndim``, point coordinates, cell connectivity of one ``GeoKind``); pmsim passes them to
``ElementSolid::new`` (reference ``src/fem/element_solid.rs:47-92``).  Node ordering per
kind follows the reference's mesh files: Qua8 corners counter-clockwise then mid-edges
0-1, 1-2, 2-3, 3-0 (``data/results/artificial/artificial-elastic-2d-qua8-mesh.msh``);
Hex8 bottom face then top face (``data/results/artificial/artificial-elastic-3d-mesh.msh``);
Hex20 corners, bottom mid-edges, top mid-edges, vertical mid-edges
(``src/base/sample_meshes.rs:541-625``).

Global DOF numbering of a solid-only mesh is ``eq = ndim*point + d`` with d = Ux, Uy, Uz
(``src/base/all_dofs.rs:87-116``; local layout ``[ux0, uy0, (uz0), ux1, ...]``,
``src/base/element_dofs.rs:123-129``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Element kinds; the integers are part of the C ABI (include/pms.h, enum pms_kind).
TRI3, TRI6, QUA4, QUA8, QUA9, TET4, TET10, HEX8, HEX20, TRI10, TRI15 = range(11)
KIND_NAMES = ["tri3", "tri6", "qua4", "qua8", "qua9", "tet4", "tet10", "hex8", "hex20", "tri10", "tri15"]
KIND_NNODE = [3, 6, 4, 8, 9, 4, 10, 8, 20, 10, 15]
KIND_NDIM = [2, 2, 2, 2, 2, 3, 3, 3, 3, 2, 2]
DEFAULT_NGAUSS = [3, 3, 4, 9, 9, 4, 4, 8, 27, 6, 12]

# Barycentric positions (multiples of 1/order, order = 3 or 4) of the nodes of the cubic and quartic
# triangles, in the node order of the reference's meshes: corners, then (Tri15) the mid-edge nodes of
# edges 0-1, 1-2, 2-0, then the edge nodes nearer the first and then the second corner of each edge,
# then the interior nodes.  The Tri15 order is pinned by src/base/sample_meshes.rs:305-362
# (smith_example_5d7_tri15); the Tri10 order follows the same pattern (not pinned by reference data).
TRI10_NODES = [(3, 0, 0), (0, 3, 0), (0, 0, 3), (2, 1, 0), (1, 2, 0), (0, 2, 1), (0, 1, 2), (1, 0, 2), (2, 0, 1),
               (1, 1, 1)]
TRI15_NODES = [(4, 0, 0), (0, 4, 0), (0, 0, 4), (2, 2, 0), (0, 2, 2), (2, 0, 2), (3, 1, 0), (1, 3, 0), (0, 3, 1),
               (0, 1, 3), (1, 0, 3), (3, 0, 1), (2, 1, 1), (1, 2, 1), (1, 1, 2)]


def kind_from_name(name: str) -> int:
    return KIND_NAMES.index(name.lower())


@dataclass
class Mesh:
    """Homogeneous mesh: every cell has the same kind."""

    ndim: int
    coords: np.ndarray  # (npoint, ndim) float64
    cells: np.ndarray  # (ncell, nnode) int64
    kind: int

    def __post_init__(self):
        self.coords = np.ascontiguousarray(self.coords, dtype=np.float64)
        self.cells = np.ascontiguousarray(self.cells, dtype=np.int64)
        if self.coords.ndim != 2 or self.coords.shape[1] != self.ndim:
            raise ValueError("coords must be (npoint, ndim)")
        if self.cells.ndim != 2 or self.cells.shape[1] != KIND_NNODE[self.kind]:
            raise ValueError("cells must be (ncell, nnode) for the given kind")
        if KIND_NDIM[self.kind] != self.ndim:
            raise ValueError("kind does not match ndim")

    @property
    def npoint(self) -> int:
        return self.coords.shape[0]

    @property
    def ncell(self) -> int:
        return self.cells.shape[0]

    @property
    def nnode(self) -> int:
        return self.cells.shape[1]

    @property
    def ndof(self) -> int:
        return self.npoint * self.ndim

    def points_where(self, pred) -> np.ndarray:
        """Sorted ids of points whose coordinates satisfy ``pred(x, y[, z])`` (vectorised)."""
        cols = [self.coords[:, i] for i in range(self.ndim)]
        return np.nonzero(pred(*cols))[0].astype(np.int64)


def _grid_ids(keep: np.ndarray) -> np.ndarray:
    ids = -np.ones(keep.shape, dtype=np.int64)
    ids[keep] = np.arange(int(keep.sum()), dtype=np.int64)
    return ids


def _higher_triangles(kind, nx, ny, lx, ly, x0, y0) -> Mesh:
    """Tri10/Tri15 rectangle: each grid square split into two triangles (a, b, c), (a, c, d) as for
    Tri3; the nodes of every triangle placed at their barycentric positions and merged by position."""
    order, table = (3, TRI10_NODES) if kind == TRI10 else (4, TRI15_NODES)
    base = structured_2d(TRI3, nx, ny, lx, ly, x0, y0)
    lam = np.array(table, dtype=np.float64) / order  # (nn, 3)
    pts = np.einsum("nk,ckd->cnd", lam, base.coords[base.cells])  # (ncell, nn, 2)
    # integer lattice coordinates (order*nx, order*ny steps) identify shared nodes exactly
    gx = np.rint((pts[..., 0] - x0) / lx * order * nx).astype(np.int64)
    gy = np.rint((pts[..., 1] - y0) / ly * order * ny).astype(np.int64)
    key = gy * (order * nx + 1) + gx
    uniq, inv = np.unique(key.ravel(), return_inverse=True)
    coords = np.stack([x0 + lx * (uniq % (order * nx + 1)) / (order * nx),
                       y0 + ly * (uniq // (order * nx + 1)) / (order * ny)], axis=1)
    return Mesh(2, coords, inv.reshape(base.ncell, len(table)), kind)


def structured_2d(kind: int, nx: int, ny: int, lx: float = 1.0, ly: float = 1.0,
                  x0: float = 0.0, y0: float = 0.0) -> Mesh:
    """Structured rectangle [x0, x0+lx] x [y0, y0+ly] of Qua4/Qua8/Qua9/Tri3/Tri6/Tri10/Tri15 cells."""
    if kind in (TRI10, TRI15):
        return _higher_triangles(kind, nx, ny, lx, ly, x0, y0)
    quad = kind in (QUA8, QUA9, TRI6)
    s = 2 if quad else 1
    ni, nj = s * nx + 1, s * ny + 1
    I, J = np.meshgrid(np.arange(ni), np.arange(nj), indexing="xy")  # (nj, ni), i fastest
    keep = np.ones((nj, ni), dtype=bool)
    if kind == QUA8:
        keep &= ~((I % 2 == 1) & (J % 2 == 1))
    ids = _grid_ids(keep)
    xs = x0 + lx * I[keep] / (s * nx)
    ys = y0 + ly * J[keep] / (s * ny)
    coords = np.stack([xs, ys], axis=1)
    ex, ey = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    ex, ey = ex.ravel(), ey.ravel()
    i0, j0 = s * ex, s * ey
    if kind == QUA4:
        cells = np.stack([ids[j0, i0], ids[j0, i0 + 1], ids[j0 + 1, i0 + 1], ids[j0 + 1, i0]], axis=1)
    elif kind in (QUA8, QUA9):
        lst = [ids[j0, i0], ids[j0, i0 + 2], ids[j0 + 2, i0 + 2], ids[j0 + 2, i0],
               ids[j0, i0 + 1], ids[j0 + 1, i0 + 2], ids[j0 + 2, i0 + 1], ids[j0 + 1, i0]]
        if kind == QUA9:
            lst.append(ids[j0 + 1, i0 + 1])
        cells = np.stack(lst, axis=1)
    elif kind == TRI3:
        a, b, c, d = ids[j0, i0], ids[j0, i0 + 1], ids[j0 + 1, i0 + 1], ids[j0 + 1, i0]
        t1 = np.stack([a, b, c], axis=1)
        t2 = np.stack([a, c, d], axis=1)
        cells = np.stack([t1, t2], axis=1).reshape(-1, 3)
    elif kind == TRI6:
        a, b, c, d = ids[j0, i0], ids[j0, i0 + 2], ids[j0 + 2, i0 + 2], ids[j0 + 2, i0]
        mab, mbc, mcd, mda = ids[j0, i0 + 1], ids[j0 + 1, i0 + 2], ids[j0 + 2, i0 + 1], ids[j0 + 1, i0]
        mac = ids[j0 + 1, i0 + 1]
        t1 = np.stack([a, b, c, mab, mbc, mac], axis=1)
        t2 = np.stack([a, c, d, mac, mcd, mda], axis=1)
        cells = np.stack([t1, t2], axis=1).reshape(-1, 6)
    else:
        raise ValueError("2D kind required")
    return Mesh(2, coords, cells, kind)


def structured_3d(kind: int, nx: int, ny: int, nz: int, lx: float = 1.0, ly: float = 1.0, lz: float = 1.0,
                  x0: float = 0.0, y0: float = 0.0, z0: float = 0.0) -> Mesh:
    """Structured box of Hex8/Hex20/Tet4 cells (Tet4: six tetrahedra per hexahedron)."""
    s = 2 if kind == HEX20 else 1
    ni, nj, nk = s * nx + 1, s * ny + 1, s * nz + 1
    K, J, I = np.meshgrid(np.arange(nk), np.arange(nj), np.arange(ni), indexing="ij")  # i fastest
    keep = np.ones((nk, nj, ni), dtype=bool)
    if kind == HEX20:
        keep &= ((I % 2) + (J % 2) + (K % 2)) <= 1
    ids = _grid_ids(keep)
    coords = np.stack([x0 + lx * I[keep] / (s * nx), y0 + ly * J[keep] / (s * ny),
                       z0 + lz * K[keep] / (s * nz)], axis=1)
    ez, ey, ex = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ex, ey, ez = ex.ravel(), ey.ravel(), ez.ravel()
    i0, j0, k0 = s * ex, s * ey, s * ez
    h = s
    corners = [ids[k0, j0, i0], ids[k0, j0, i0 + h], ids[k0, j0 + h, i0 + h], ids[k0, j0 + h, i0],
               ids[k0 + h, j0, i0], ids[k0 + h, j0, i0 + h], ids[k0 + h, j0 + h, i0 + h], ids[k0 + h, j0 + h, i0]]
    if kind == HEX8:
        cells = np.stack(corners, axis=1)
    elif kind == HEX20:
        mids = [ids[k0, j0, i0 + 1], ids[k0, j0 + 1, i0 + 2], ids[k0, j0 + 2, i0 + 1], ids[k0, j0 + 1, i0],
                ids[k0 + 2, j0, i0 + 1], ids[k0 + 2, j0 + 1, i0 + 2], ids[k0 + 2, j0 + 2, i0 + 1],
                ids[k0 + 2, j0 + 1, i0],
                ids[k0 + 1, j0, i0], ids[k0 + 1, j0, i0 + 2], ids[k0 + 1, j0 + 2, i0 + 2], ids[k0 + 1, j0 + 2, i0]]
        cells = np.stack(corners + mids, axis=1)
    elif kind == TET4:
        c = corners
        # six tetrahedra around the 0-6 diagonal, all positively oriented
        tets = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]
        cells = np.stack([np.stack([c[a], c[b], c[cc], c[d]], axis=1) for (a, b, cc, d) in tets],
                         axis=1).reshape(-1, 4)
    else:
        raise ValueError("3D kind required")
    return Mesh(3, coords, cells, kind)


def read_msh(path: str) -> Mesh:
    """Reads the reference's plain-text mesh format (header, points, cells; '#' comments)."""
    lines = [ln for ln in open(path).read().split("\n") if ln.strip() and not ln.lstrip().startswith("#")]
    ndim, npoint, ncell = map(int, lines[0].split())
    coords = np.array([[float(v) for v in ln.split()[2:2 + ndim]] for ln in lines[1:1 + npoint]])
    rows = [ln.split() for ln in lines[1 + npoint:1 + npoint + ncell]]
    kinds = {r[2] for r in rows}
    if len(kinds) != 1:
        raise ValueError("only homogeneous meshes are supported")
    kind = kind_from_name(kinds.pop())
    cells = np.array([[int(v) for v in r[3:]] for r in rows], dtype=np.int64)
    return Mesh(ndim, coords, cells, kind)
