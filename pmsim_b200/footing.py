"""Synthetic plane-strain strip-footing problems used by the benchmarks and tests.

The footing: a 10 m x 5 m rectangle of Qua8 cells with 3x3 Gauss points, von Mises (nu = 0.3,
H = 0), bottom fixed, sides on rollers, and the top nodes with x <= width pushed down by
0.005 m per unit load step (10 steps to 0.05 m), solved with Lagrange multipliers
(``Config::set_lagrange_mult_method`` / ``set_incremental``, reference ``src/base/config.rs``).
The default instance is the 20 x 10 mesh with E = 1e4 kPa, z0 = 9 kPa and width 1 m; the batched
population draws nx in [8, 64], ny in [4, 32], E log-normal (median 1e4, sigma_log 0.5), z0 in
[5, 20] and width in [0.5, 2] from one seed.
"""
from __future__ import annotations

import numpy as np

from . import mesh as M
from .batch import Problem
from .elements import Material

LX, LY = 10.0, 5.0
STEP_UY = -0.005


def footing_problem(nx=20, ny=10, young=1e4, z_ini=9.0, width=1.0, nsteps=10, poisson=0.3, hh=0.0) -> Problem:
    m = M.structured_2d(M.QUA8, nx, ny, LX, LY)
    tol = 1e-8
    ess = []
    for p in m.points_where(lambda x, y: np.abs(y) < tol):
        ess += [(2 * p, 0.0, None), (2 * p + 1, 0.0, None)]
    for p in m.points_where(lambda x, y: (np.abs(x) < tol) | (np.abs(x - LX) < tol)):
        ess += [(2 * p, 0.0, None)]
    for p in m.points_where(lambda x, y: (np.abs(y - LY) < tol) & (x <= width + tol)):
        ess += [(2 * p + 1, STEP_UY, _linear)]
    return Problem(m, Material.von_mises(young, poisson, hh, z_ini), ess, nsteps=nsteps, ngauss=9,
                   name=f"footing {nx}x{ny} E={young:.4g} z0={z_ini:.3g} B={width:.3g}",
                   meta=dict(nx=nx, ny=ny, young=young, z_ini=z_ini, width=width))


def _linear(t):
    return t


def population(n, seed=2024, nsteps=10):
    """n footings drawn from the batched configuration's distributions (one seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx = int(rng.integers(8, 65))
        ny = int(rng.integers(4, 33))
        young = float(1e4 * np.exp(rng.normal(0.0, 0.5)))
        z0 = float(rng.uniform(5.0, 20.0))
        width = float(rng.uniform(0.5, 2.0))
        out.append(footing_problem(nx, ny, young, z0, width, nsteps=nsteps))
    return out


def block_problem(nx=8, ny=8, nz=8, young=1e4, z_ini=9.0, nsteps=10, poisson=0.3, hh=0.0) -> Problem:
    """3D block of Hex8 cells (unit cell size), base fixed, the central quarter of the top face
    pressed down to 0.5% of the height over nsteps unit load steps."""
    m = M.structured_3d(M.HEX8, nx, ny, nz, float(nx), float(ny), float(nz))
    tol = 1e-8
    ess = []
    for p in m.points_where(lambda x, y, z: np.abs(z) < tol):
        ess += [(3 * p, 0.0, None), (3 * p + 1, 0.0, None), (3 * p + 2, 0.0, None)]
    cx, cy = nx / 2.0, ny / 2.0
    top = m.points_where(lambda x, y, z: (np.abs(z - nz) < tol) & (np.abs(x - cx) <= nx / 4.0 + tol)
                         & (np.abs(y - cy) <= ny / 4.0 + tol))
    per_step = -0.005 * nz / nsteps
    for p in top:
        ess += [(3 * p + 2, per_step, _linear)]
    return Problem(m, Material.von_mises(young, poisson, hh, z_ini), ess, nsteps=nsteps, ngauss=8,
                   name=f"block {nx}x{ny}x{nz} E={young:.4g} z0={z_ini:.3g}",
                   meta=dict(nx=nx, ny=ny, nz=nz, young=young, z_ini=z_ini))


def request_population(n, seed=7, nsteps=10):
    """Requests of the served configuration: 70% Qua8 footings with 1k-50k DOF, 30% Hex8 blocks
    with nx, ny, nz in [8, 40] (up to 206,763 DOF); E log-normal (median 1e4, sigma_log 0.5) and
    z0 in [5, 20] as in the batched population."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        young = float(1e4 * np.exp(rng.normal(0.0, 0.5)))
        z0 = float(rng.uniform(5.0, 20.0))
        if rng.random() < 0.7:
            # footing 10 m x 5 m with nx = 2 ny: ndof ~ 6 nx ny spans 1k..50k
            ndof_target = float(np.exp(rng.uniform(np.log(1e3), np.log(5e4))))
            ny = max(4, int(round(np.sqrt(ndof_target / 12.0))))
            nx = 2 * ny
            width = float(rng.uniform(0.5, 2.0))
            out.append(footing_problem(nx, ny, young, z0, width, nsteps=nsteps))
        else:
            nx, ny, nz = (int(v) for v in rng.integers(8, 41, size=3))
            out.append(block_problem(nx, ny, nz, young, z0, nsteps=nsteps))
    return out
