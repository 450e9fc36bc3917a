"""Host-made inputs that drive the element path into the reference's error returns.

The von Mises return map with softening H = -3G/2 gives sigma_d_new = 2 z - sigma_d_trial exactly,
so a uniform pure shear with sigma_d_trial = 2 z ends on a zero deviator ("von Mises plastic update
must not lead to zero sigma_d", src/material/von_mises.rs:212-216), and one with
sigma_d_trial = 2 z - 1.1e-10 ends on sigma_d = 1.1e-10: the update passes (>= 1e-10) but the
tangent refuses (norm_s = sqrt(2/3) sigma_d < 1e-10, von_mises.rs:147-150).  A displacement field
u_x = gamma * y on the nodes with x in a band gives that uniform shear on the cells inside the band
(pure shear: sigma_d = sqrt(3) G gamma) and no error elsewhere.
"""
import numpy as np

from pmsim_b200 import mesh as M

E, NU, Z0 = 2e5, 0.3, 250.0
G = E / (2.0 * (1.0 + NU))
H_SOFT = -1.5 * G
GAMMA_ZERO_SIGMA_D = 2.0 * Z0 / (np.sqrt(3.0) * G)
GAMMA_ZERO_NORM_S = (2.0 * Z0 - 1.1e-10) / (np.sqrt(3.0) * G)


def shear_mesh(kind):
    if M.KIND_NDIM[kind] == 2:
        return M.structured_2d(kind, 8, 3, 8.0, 3.0)
    return M.structured_3d(kind, 6, 2, 2, 6.0, 2.0, 2.0)


def band_shear(mesh, bands):
    """ddu with u_x = gamma * y on the nodes with x0 <= x <= x1 for each (x0, x1, gamma)."""
    u = np.zeros((mesh.npoint, mesh.ndim))
    x, y = mesh.coords[:, 0], mesh.coords[:, 1]
    for x0, x1, gamma in bands:
        sel = (x >= x0 - 1e-12) & (x <= x1 + 1e-12)
        u[sel, 0] = gamma * y[sel]
    return u.reshape(-1).copy()


def cells_inside(mesh, x0, x1):
    """Cells whose nodes all lie in x0 <= x <= x1 (uniform shear there)."""
    x = mesh.coords[mesh.cells, 0]
    return np.flatnonzero(np.all((x >= x0 - 1e-12) & (x <= x1 + 1e-12), axis=1))


def inverted(mesh, cell):
    """The mesh with one cell's nodes in reflected order (negative Jacobian determinant)."""
    cells = mesh.cells.copy()
    if mesh.ndim == 2:
        nc = {M.QUA4: 4, M.QUA8: 4, M.QUA9: 4, M.TRI3: 3, M.TRI6: 3}[mesh.kind]
        corner = cells[cell, :nc][::-1].copy()
        # corners reversed: the mid-edge node of edge (k, k+1) becomes that of edge (nc-2-k, nc-1-k)
        mids = cells[cell, nc:2 * nc].copy() if cells.shape[1] >= 2 * nc else None
        cells[cell, :nc] = corner
        if mids is not None:
            cells[cell, nc:2 * nc] = np.roll(mids[::-1], -1)
    else:
        raise ValueError("2D only")
    return M.Mesh(mesh.ndim, mesh.coords, cells, mesh.kind)
