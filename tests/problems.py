"""Golden problems of the reference's integration tests, rebuilt from the fixtures.

Each builder returns (mesh, model, params, ngauss, essential, nsteps, golden, tolerances) in
the form the oracle driver and the product solver both take.  The boundary conditions and
material constants restate the reference tests cited on each builder.
"""
import os

import numpy as np

from pmsim_b200.mesh import Mesh, QUA4, QUA8, kind_from_name

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-8  # coordinate match, as gemlab's At::X / At::Y searches


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def _ess(points, dof, ndim, const=0.0, fn=None):
    return [(ndim * int(p) + dof, const, fn) for p in points]


def single_element_2d():
    """tests/test_von_mises_single_element_2d.rs: Qua4, 1 IP, E=1500, nu=0.25, H=800, z0=9."""
    g = load("spo_single_element_2d.npz")
    m = Mesh(2, np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]]), np.array([[0, 1, 2, 3]]), QUA4)
    E, nu, z0 = 1500.0, 0.25, 9.0
    dy = z0 * (1.0 - nu * nu) / (E * np.sqrt(1.0 - nu + nu * nu))
    ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y) < TOL), 1, 2)
           + _ess(m.points_where(lambda x, y: abs(y - 1.0) < TOL), 1, 2, 1.0, lambda t: -dy * t))
    return dict(mesh=m, params=(E, nu, 800.0, z0), ngauss=1, essential=ess, nsteps=5, golden=g,
                tol_u=1e-13, tol_s=1e-10, sym_tol=1e-10)


def two_by_two_2d():
    """tests/test_von_mises_2x2_elements_2d.rs: four Qua8, 4 IP, same material as above."""
    g = load("spo_2x2_elements_2d.npz")
    m = Mesh(2, g["coords"], g["cells"], QUA8)
    E, nu, z0 = 1500.0, 0.25, 9.0
    dy = z0 * (1.0 - nu * nu) / (E * np.sqrt(1.0 - nu + nu * nu))
    ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y) < TOL), 1, 2)
           + _ess(m.points_where(lambda x, y: abs(y - 2.0) < TOL), 1, 2, 1.0, lambda t: -dy * t))
    return dict(mesh=m, params=(E, nu, 800.0, z0), ngauss=4, essential=ess, nsteps=5, golden=g,
                tol_u=1e-12, tol_s=1e-9, sym_tol=1e-10)


UY_754 = [0.0, -0.01, -0.015, -0.02, -0.025, -0.035, -0.045, -0.055, -0.065, -0.075, -0.08, -0.09, -0.11,
          -0.14, -0.2]


def footing_754():
    """tests/test_spo_754_footing.rs: Qua8 mesh, 4 IP, E=1e7, nu=0.48, z0=848.7, H=0, 14 steps."""
    g = load("spo_754_footing.npz")
    m = Mesh(2, g["coords"], g["cells"], QUA8)
    ess = (_ess(m.points_where(lambda x, y: (abs(x) < TOL) | (abs(x - 500.0) < TOL)), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y) < TOL), 1, 2)
           + _ess(m.points_where(lambda x, y: (abs(y - 500.0) < TOL) & (x <= 50.0)), 1, 2, 1.0,
                  lambda t: UY_754[int(t)]))
    return dict(mesh=m, params=(1e7, 0.48, 0.0, 848.7), ngauss=4, essential=ess, nsteps=14, golden=g,
                tol_u=1e-10, tol_s=5e-5, sym_tol=1e-5)


UY_755 = [0.0, 0.005, 0.01, 0.015, 0.02, 0.03, 0.04, 0.05, 0.07, 0.09, 0.11, 0.115, 0.12, 0.13, 0.15, 0.17]


def tensile_755():
    """tests/test_spo_755_tensile.rs: Qua8 mesh, 4 IP, E=206.9, nu=0.29, z0=0.45, H=0, 15 steps."""
    g = load("spo_755_tensile.npz")
    m = Mesh(2, g["coords"], g["cells"], QUA8)
    ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: (abs(y) < TOL) & (x < 0.50001)), 1, 2)
           + _ess(m.points_where(lambda x, y: abs(y - 15.0) < TOL), 1, 2, 1.0, lambda t: UY_755[int(t)]))
    return dict(mesh=m, params=(206.9, 0.29, 0.0, 0.45), ngauss=4, essential=ess, nsteps=15, golden=g,
                tol_u=1e-7, tol_s=1.2e-5, sym_tol=1e-5)


SPO_PROBLEMS = {"single_element_2d": single_element_2d, "2x2_elements_2d": two_by_two_2d,
                "footing_754": footing_754, "tensile_755": tensile_755}


def smith_5d11():
    """tests/test_solid_smith_5d11_qua4_plane_strain_uy.rs: linear elastic Qua4, LMM, one step."""
    g = load("smith_5d11_qua4.npz")
    m = Mesh(2, g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(x - 30.0) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y + 10.0) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y + 10.0) < TOL), 1, 2)
           + _ess(m.points_where(lambda x, y: (abs(y) < TOL) & (x <= 10.0)), 1, 2, -1e-5))
    return dict(mesh=m, params=(1e6, 0.3, 0.0, 1.0), ngauss=0, essential=ess, nsteps=1, golden=g)


def compare_step(golden, step, u, sig, ngauss_ref):
    """Max abs differences (displacement, Mandel stress) as src/util/compare_results.rs:42-155."""
    gu = golden["displacement"][step].reshape(-1)
    gs = np.array(golden["stresses"][step], dtype=float)
    gs[..., 3:] *= np.sqrt(2.0)
    s = sig.reshape(gs.shape)
    return float(np.max(np.abs(u - gu))), float(np.max(np.abs(s - gs)))
