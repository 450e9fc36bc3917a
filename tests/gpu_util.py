"""Helpers shared by the GPU parity tests: seeded meshes/states and normwise comparisons."""
import numpy as np

from pmsim_b200 import mesh as M

TOL = 1e-12  # relative, normwise: |a - b|_max <= TOL * |b|_max (FP64 parity bar)


def assert_close(a, b, tol=TOL, what=""):
    a = np.asarray(a, dtype=float)
    b = np.asarray(b, dtype=float)
    assert a.shape == b.shape, (what, a.shape, b.shape)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    err = float(np.max(np.abs(a - b))) if a.size else 0.0
    assert err <= tol * scale, f"{what}: max|diff| = {err:.3e} > {tol:.0e} * {scale:.3e}"
    return err / scale


def perturbed_mesh(kind, seed=0, n=(3, 2, 2), amp=0.08):
    """Structured mesh with interior nodes moved randomly (general element geometry)."""
    if M.KIND_NDIM[kind] == 2:
        m = M.structured_2d(kind, n[0], n[1], float(n[0]), float(n[1]))
    else:
        m = M.structured_3d(kind, n[0], n[1], n[2], float(n[0]), float(n[1]), float(n[2]))
    rng = np.random.default_rng(seed)
    if kind in (M.TRI10, M.TRI15):  # nodes 1/3 or 1/4 of a cell apart: move them less
        amp *= 0.4
    c = m.coords.copy()
    lo, hi = c.min(0), c.max(0)
    interior = np.all((c > lo + 1e-9) & (c < hi - 1e-9), axis=1)
    c[interior] += rng.uniform(-amp, amp, size=(int(interior.sum()), m.ndim))
    return M.Mesh(m.ndim, c, m.cells, kind)


def plastic_ddu(mesh, seed=0, strain=1.2e-3):
    """Smooth displacement increment (compression + shear) plus noise: mixes elastic and plastic IPs
    for E=2e5, z0=250."""
    rng = np.random.default_rng(seed)
    x = mesh.coords
    u = np.zeros_like(x)
    u[:, -1] = -strain * x[:, -1]
    u[:, 0] = 0.6 * strain * x[:, -1] * (1 + 0.3 * np.sin(x[:, 0]))
    u += rng.normal(0, 0.4 * strain, size=x.shape)
    return u.reshape(-1).copy()
