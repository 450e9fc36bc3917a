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


def _sgm(name):
    g = load(name + ".npz")
    m = Mesh(g["coords"].shape[1], g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    return g, m


def sgm_natural(case):
    """Linear-elastic Smith-Griffiths runs with natural boundary conditions (reduced-system method,
    one step), from tests/test_solid_smith_5d{2,7,15,27,30,24}_*.rs."""
    from pmsim_b200.natural import Natural, find_sides
    if case == "5d2_tri3":
        g, m = _sgm("smith_5d2_tri3")
        ess = _ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(y + 1) < TOL), 1, 2)
        nat = Natural(m).sides(find_sides(m, lambda p: abs(p[1]) < TOL), -1.0)
        return dict(mesh=m, mats=[(1e6, 0.3)], cmat=None, ngauss=0, essential=ess, natural=nat, golden=g, tol=1e-15)
    if case in ("5d15_qua8", "5d27_qua9"):
        g, m = _sgm("smith_" + case)
        ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(x - 6) < TOL), 0, 2)
               + _ess(m.points_where(lambda x, y: abs(y + 9) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(y + 9) < TOL), 1, 2))
        nat = Natural(m).sides(find_sides(m, lambda p: abs(p[1]) < TOL, lambda p: p[0] <= 3.0 + TOL), -1.0)
        return dict(mesh=m, mats=[(1e6, 0.3)], cmat=None, ngauss=4 if case == "5d15_qua8" else 0, essential=ess,
                    natural=nat, golden=g, tol=1e-12 if case == "5d15_qua8" else 3e-13)
    if case == "5d7_tri15":  # tests/test_solid_smith_5d7_tri15_plane_strain.rs (12 IP, point loads)
        g, m = _sgm("smith_5d7_tri15")
        ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(x - 6) < TOL), 0, 2)
               + _ess(m.points_where(lambda x, y: abs(y + 2) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(y + 2) < TOL), 1, 2))
        nat = (Natural(m).points([0, 20], 1, -0.0778).points([5, 15], 1, -0.3556).points([10], 1, -0.1333))
        return dict(mesh=m, mats=[(1e5, 0.2)], cmat=None, ngauss=12, essential=ess, natural=nat, golden=g, tol=1e-11)
    if case == "5d30_tet4":
        g, m = _sgm("smith_5d30_tet4")
        ess = (_ess(m.points_where(lambda x, y, z: abs(x) < TOL), 0, 3) + _ess(m.points_where(lambda x, y, z: abs(y) < TOL), 1, 3)
               + _ess(m.points_where(lambda x, y, z: abs(z + 1) < TOL), 2, 3))
        nat = Natural(m).points([0, 5], 2, -0.1667).points([1, 4], 2, -0.3333)
        return dict(mesh=m, mats=[(100.0, 0.3)], cmat=None, ngauss=0, essential=ess, natural=nat, golden=g, tol=1e-15)
    if case == "5d24_hex20":
        g, m = _sgm("smith_5d24_hex20")
        ess = (_ess(m.points_where(lambda x, y, z: abs(x) < TOL), 0, 3) + _ess(m.points_where(lambda x, y, z: abs(y) < TOL), 1, 3))
        for d in range(3):
            ess += _ess(m.points_where(lambda x, y, z: abs(z + 2) < TOL), d, 3)
        nat = Natural(m).sides(find_sides(m, lambda p: abs(p[2]) < TOL, lambda p: p[1] <= 1.0 + TOL), -1.0)
        cmat = (g["attribute"] - 1).astype(np.int32)
        return dict(mesh=m, mats=[(100.0, 0.3), (50.0, 0.3)], cmat=cmat, ngauss=8, essential=ess, natural=nat, golden=g,
                    tol=2e-9)
    raise KeyError(case)


SGM_NATURAL = ["5d2_tri3", "5d7_tri15", "5d15_qua8", "5d27_qua9", "5d30_tet4", "5d24_hex20"]

P_751 = [0.0, 0.1, 0.14, 0.18, 0.19, 0.192]


def pres_cylin_751():
    """tests/test_spo_751_pres_cylin.rs: Qua8 ring, 4 IP, E=210, nu=0.3, z0=0.24, H=0, internal pressure
    on the inner circle (r = 100), reduced-system method, tol_mdu_rel = 1e-10, 5 steps."""
    from pmsim_b200.natural import Natural, find_sides
    g = load("spo_751_pres_cylin.npz")
    m = Mesh(2, g["coords"], g["cells"], QUA8)
    ess = _ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(y) < TOL), 1, 2)
    on_circle = lambda p: abs(np.hypot(p[0], p[1]) - 100.0) < 1e-6  # noqa: E731
    nat = Natural(m).sides(find_sides(m, on_circle), 1.0, lambda t: -P_751[int(t)])
    # tol_s: the reference test's 1e-14 (absolute, on stresses up to 0.26) is ~40 ulps, the rounding
    # noise of the linear solve; 2e-14 (1e-13 relative) keeps this pin well inside the 1e-12 parity bar.
    # iterations: pmsim's own Newton history of this run (data/log-nonlin-tests.txt, SPO-751 block).
    return dict(mesh=m, params=(210.0, 0.3, 0.0, 0.24), ngauss=4, essential=ess, natural=nat, nsteps=5, golden=g,
                tol_u=1e-11, tol_s=2e-14, iterations=[2, 5, 6, 5, 9])


P_753 = [0.0, 100.0, 200.0, 220.0, 230.0, 240.0, 250.0, 255.0, 257.0, 259.0, 259.5, 259.75, 259.77]


def circ_plate_753():
    """tests/test_spo_753_circ_plate.rs: axisymmetric circular plate (radius 10, thickness 1), 10 Qua8
    cells, 4 IP, von Mises E=1e7, nu=0.24, z0=16000, H=0; u_r = 0 on the axis (x = 0), u_z = 0 at
    the rim corner (10, 0); normal pressure P(t) on the top face (y = 1) up to 259.77, near the
    collapse load; Lagrange multipliers, 12 load steps, at most 20 iterations each.  Tolerances as
    in the reference test: 1e-9 on displacements, 1e-6 on stresses."""
    from pmsim_b200.natural import Natural, find_sides
    g = load("spo_753_circ_plate.npz")
    m = Mesh(2, g["coords"], g["cells"], QUA8)
    ess = _ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + \
        _ess(m.points_where(lambda x, y: (np.abs(x - 10.0) < TOL) & (np.abs(y) < TOL)), 1, 2)
    nat = Natural(m, axisymmetric=True).sides(find_sides(m, lambda p: abs(p[1] - 1.0) < TOL), 1.0,
                                              lambda t: -P_753[int(t)])
    return dict(mesh=m, params=(1e7, 0.24, 0.0, 16000.0), ngauss=4, essential=ess, natural=nat, nsteps=12,
                golden=g, tol_u=1e-9, tol_s=1e-6)


P_752 = [0.0, 0.15, 0.3, 0.33, 0.33269]


def pres_sphere_752():
    """tests/test_spo_752_pres_sphere.rs (the collapse run): the SPO 7.5.1 Qua8 mesh taken as an
    axisymmetric section of a thick sphere (inner radius 100, outer 200), 4 IP, von Mises E=210,
    nu=0.3, z0=0.24, H=0, u_r = 0 on the axis (x = 0), u_z = 0 on the equator (y = 0), internal
    pressure up to 0.33269 (near collapse), Lagrange multipliers, 4 load steps.  The reference test's
    tolerances are loose (4.33e-2 on displacements, 2.55e-2 on stresses) because the HYPLAS data
    were computed differently; they are the reference's."""
    from pmsim_b200.natural import Natural, find_sides
    gm = load("spo_751_pres_cylin.npz")
    g = load("spo_752_pres_sphere_collapse.npz")
    m = Mesh(2, gm["coords"], gm["cells"], QUA8)
    ess = _ess(m.points_where(lambda x, y: np.abs(x) < TOL), 0, 2) + \
        _ess(m.points_where(lambda x, y: np.abs(y) < TOL), 1, 2)
    on_circle = lambda p: abs(np.hypot(p[0], p[1]) - 100.0) < 1e-6  # noqa: E731
    nat = Natural(m, axisymmetric=True).sides(find_sides(m, on_circle), 1.0, lambda t: -P_752[int(t)])
    return dict(mesh=m, params=(210.0, 0.3, 0.0, 0.24), ngauss=4, essential=ess, natural=nat, nsteps=4,
                golden=g, tol_u=4.33e-2, tol_s=2.55e-2)


class MultiMaterialOracle:
    """The oracle's element calls over a mesh whose cells use several materials: one homogeneous
    OracleElements per material on its subset of cells (all points kept), summed like the
    reference's Elements loop over cells (src/fem/elements.rs:132-163)."""

    def __init__(self, mesh, cmat, mats, ngauss=0, axisymmetric=False):
        import oracle
        self.groups = []
        for k, (E, nu) in enumerate(mats):
            sub = Mesh(mesh.ndim, mesh.coords, mesh.cells[cmat == k], mesh.kind)
            self.groups.append(oracle.OracleElements(sub, 0, oracle.Params(E, nu, 0.0, 1.0), ngauss=ngauss,
                                                     axisymmetric=axisymmetric))
        self.ndof = mesh.ndof

    def _each(self, name, *a):
        for g in self.groups:
            getattr(g, name)(*a)

    def initialize(self):
        self._each("initialize")

    def reset_algorithmic_variables(self):
        self._each("reset_algorithmic_variables")

    def backup_secondary_values(self):
        self._each("backup_secondary_values")

    def restore_secondary_values(self):
        self._each("restore_secondary_values")

    def update_secondary_values(self, ddu):
        self._each("update_secondary_values", ddu)

    def assemble_f_int(self):
        return sum(g.assemble_f_int() for g in self.groups)

    def assemble_kk_csr(self):
        import scipy.sparse as sp
        k = None
        for g in self.groups:
            ip, ix, v = g.assemble_kk_csr()
            m = sp.csr_matrix((v, ix, ip), shape=(self.ndof, self.ndof))
            k = m if k is None else k + m
        k = k.tocsr()
        k.sort_indices()
        return k.indptr, k.indices, k.data


def sgm_5d17_axisym():
    """tests/test_solid_smith_5d17_qua4_axisym.rs: axisymmetric Qua4 (9 IP), two linear-elastic layers
    (E=100, nu=0.3 on top; E=1000, nu=0.45 below), sides and base on rollers/fixed, point loads Fy on
    points 0, 3, 6; reduced-system method, one step."""
    g = load("smith_5d17_qua4_axisym.npz")
    m = Mesh(2, g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    ess = (_ess(m.points_where(lambda x, y: abs(x) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(x - 30) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: abs(y + 10) < TOL), 0, 2) + _ess(m.points_where(lambda x, y: abs(y + 10) < TOL), 1, 2))
    loads = [(2 * 0 + 1, -2.6667), (2 * 3 + 1, -23.3333), (2 * 6 + 1, -24.0)]
    return dict(mesh=m, mats=[(100.0, 0.3), (1000.0, 0.45)], cmat=(g["attribute"] - 1).astype(np.int32), ngauss=9,
                essential=ess, loads=loads, golden=g)


def bhatti_1d6_plane_stress():
    """tests/test_solid_bhatti_1d6_plane_stress.rs: Tri3 bracket in plane stress (thickness 0.25),
    linear elastic E=1e4, nu=0.2, points 0 and 1 fixed, Qn = -20 on the top sides (1,3) and (3,5)."""
    from pmsim_b200.natural import Natural, find_sides
    g = load("bhatti_1d6_plane_stress.npz")
    m = Mesh(2, g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    ess = [(2 * p + d, 0.0, None) for p in (0, 1) for d in range(2)]
    top = find_sides(m, lambda p: abs(p[1] - (2.0 - p[0] / 4.0)) < TOL)
    nat = Natural(m, thickness=0.25).sides(top, -20.0)
    return dict(mesh=m, young=1e4, poisson=0.2, thickness=0.25, essential=ess, natural=nat, golden=g, nsides=len(top))


def felippa_thick_cylinder():
    """tests/test_solid_felippa_thick_cylinder_axisym.rs (Felippa, A-FEM benchmark 14.1): two
    axisymmetric Qua8 (r from 4 to 10, height 2), 4 IP, linear elastic E=1000, nu=0; u_z = 0 on the
    bottom and top edges, Qn = -10 (internal pressure) on the inner edge r = 4; one step.  The test
    checks u_r at the points of y = 0 against the thick-cylinder solution (Felippa's eq. 14.2) to
    1e-15."""
    from pmsim_b200.natural import Natural, find_sides
    g = load("felippa_thick_cylinder_axisym.npz")
    m = Mesh(2, g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    rin, rout, pres, young, nu = 4.0, 10.0, 10.0, 1000.0, 0.0
    ess = _ess(m.points_where(lambda x, y: (np.abs(y) < TOL) | (np.abs(y - 2.0) < TOL)), 1, 2)
    nat = Natural(m, axisymmetric=True).sides(find_sides(m, lambda p: abs(p[0] - rin) < TOL), -pres)

    def ur(r):
        return pres * (rin * rin * (1.0 + nu) * (rout * rout + r * r * (1.0 - 2.0 * nu))) / (
            young * (rout * rout - rin * rin) * r)

    return dict(mesh=m, young=young, poisson=nu, ngauss=4, essential=ess, natural=nat,
                check_points=m.points_where(lambda x, y: np.abs(y) < TOL), ur=ur, tol=1e-15)


def strip_load_stress(x, y, bb, hh, qn, nu):
    """Flexible strip footing of half-width bb on an elastic half-plane (Davis and Selvadurai,
    Elasticity and Geomechanics, 1996, p. 138), as src/analytical/elast_plane_strain_flexible_foot.rs:52-80
    states it: the surface is y = hh, z = hh - y the depth; returns (s_xx, s_yy, s_xy)."""
    z = hh - y
    d1, d2 = x - bb, bb + x
    s = np.sign(d1)
    if z == 0.0:
        th1, th2 = s * np.pi / 2.0, np.pi / 2.0
    else:
        th1, th2 = s * np.arctan(abs(d1) / z), np.arctan(d2 / z)
    s1, s2 = np.sin(2.0 * th1), np.sin(2.0 * th2)
    m = -qn / np.pi
    syy = m * ((th2 + 0.5 * s2) - (th1 + 0.5 * s1))
    sxx = m * ((th2 - 0.5 * s2) - (th1 - 0.5 * s1))
    sxy = m * (s2 * s2 - s1 * s1)
    return sxx, syy, sxy


def durand_farias_example4():
    """tests/test_durand_farias_example4.rs: flexible strip footing (half-width B = 2.5) on a
    15B x 15B plane-strain Qua4 domain (49 cells), 4 IP, linear elastic E=1000, nu=0; u_x = 0 on the
    left and right edges, u_y = 0 on the bottom, Qn = -200 on the top edges with x <= B; one step.
    The test extrapolates the IP stresses of the cells on the left edge to their nodes (averaged at
    shared nodes), keeps the nodes with x below half the first cell's width and checks each against
    the strip-load solution: |s - s_ana| / Qn within 0.25 (xx), 0.23 (yy) and 0.09 (xy)."""
    from pmsim_b200.natural import Natural, find_sides
    g = load("durand_farias_example4_qua4.npz")
    m = Mesh(2, g["coords"], g["cells"], kind_from_name(str(g["kind"])))
    bb, qn = 2.5, 200.0
    ww = hh = 15.0 * bb
    ess = (_ess(m.points_where(lambda x, y: (np.abs(x) < TOL) | (np.abs(x - ww) < TOL)), 0, 2)
           + _ess(m.points_where(lambda x, y: np.abs(y) < TOL), 1, 2))
    footing = find_sides(m, lambda p: abs(p[1] - hh) < TOL, lambda p: p[0] <= bb)
    nat = Natural(m).sides(footing, -qn)
    left_cells = sorted({c for c, _ in find_sides(m, lambda p: abs(p[0]) < TOL)})
    return dict(mesh=m, young=1000.0, poisson=0.0, ngauss=4, essential=ess, natural=nat, bb=bb, hh=hh, qn=qn,
                left_cells=left_cells, tols=(0.25, 0.23, 0.09))


def nodal_stresses(mesh, cells, sig, ngauss, keep):
    """IP stresses (Mandel rows, cell-major) extrapolated to the nodes of `cells` and averaged at
    shared nodes, for the nodes whose coordinates satisfy keep(x, y), sorted by x then y
    (src/fem/post_processing.rs:617-670).  The extrapolation matrix is the least-squares inverse of
    the shape functions at the IPs; with as many IPs as nodes (Qua4, 4 IP) it is N^-1.
    Returns [(x, y, s_xx, s_yy, s_xy)]."""
    import oracle
    nn = mesh.nnode
    ksi, _ = oracle.gauss(mesh.kind, ngauss)
    nmat = np.array([oracle.shape(mesh.kind, ksi[p][:mesh.ndim])[0][:nn] for p in range(len(ksi))])
    ext = np.linalg.pinv(nmat)
    acc, cnt = {}, {}
    for c in cells:
        vals = ext @ sig[c * ngauss:(c + 1) * ngauss]
        for a, pt in enumerate(mesh.cells[c]):
            acc[int(pt)] = acc.get(int(pt), 0.0) + vals[a]
            cnt[int(pt)] = cnt.get(int(pt), 0) + 1
    out = []
    for pt in acc:
        x, y = mesh.coords[pt]
        if keep(x, y):
            v = acc[pt] / cnt[pt]
            out.append((x, y, v[0], v[1], v[3] / np.sqrt(2.0)))
    return sorted(out, key=lambda r: (r[0], r[1]))


def one_qua4_mesh():
    """gemlab's Samples::one_qua4: the unit square, nodes counter-clockwise from the origin."""
    return Mesh(2, np.array([[0.0, 0.0], [1.0, 0.0], [1.0, 1.0], [0.0, 1.0]]), np.array([[0, 1, 2, 3]]), QUA4)


def prescribe_displacements_2d():
    """tests/test_prescribe_displacements_2d.rs: one plane-strain Qua4 (default rule, 4 IP), linear
    elastic E=1500, nu=0.25; u_x = 0 on the left edge, u_y = 0 on the bottom, u_y = -0.1 on the top;
    Lagrange multipliers, one step.  Expected U: u_x = eps_x = -dy nu / (nu - 1) at the right nodes,
    u_y = -dy at the top, to 1e-15."""
    m = one_qua4_mesh()
    dy, nu = 0.1, 0.25
    ess = (_ess(m.points_where(lambda x, y: np.abs(x) < TOL), 0, 2)
           + _ess(m.points_where(lambda x, y: np.abs(y) < TOL), 1, 2)
           + _ess(m.points_where(lambda x, y: np.abs(y - 1.0) < TOL), 1, 2, -dy))
    eps_x = -dy * nu / (nu - 1.0)
    return dict(mesh=m, young=1500.0, poisson=nu, essential=ess,
                expected=np.array([0.0, 0.0, eps_x, 0.0, eps_x, -dy, 0.0, -dy]), tol=1e-15)


def solid_prescribed_displacement():
    """tests/test_solid_prescribed_displacement.rs: one plane-strain Qua4 (4 IP), linear elastic E=1,
    nu=0.25; u_x = 0 at point 0, u_y = 0 at points 0 and 1, u_y = STRAIN_Y at points 2 and 3, the
    uniaxial strain of a vertical stress q = -2.  Both of the test's approaches (partitioned system;
    residual with unit diagonal rows) must give sigma = (0, q, q nu, 0) at every IP to 1e-15; the
    residual approach also pins -R on the unknown equations (0.375, 0.375, -0.375 to six
    decimals) and dU = (0, 0, 0.625, 0, 0.625, -1.875, 0, -1.875) to 1e-15."""
    young, nu, q = 1.0, 0.25, -2.0
    strain_y = -q * (nu - 1.0) * (nu + 1.0) / young
    presc = {0: 0.0, 1: 0.0, 3: 0.0, 5: strain_y, 7: strain_y}
    return dict(mesh=one_qua4_mesh(), young=young, poisson=nu, prescribed=presc, unknown=[2, 4, 6],
                stress=np.array([0.0, q, q * nu, 0.0]), e1=np.array([0.375, 0.375, -0.375]),
                ddu=np.array([0.0, 0.0, 0.625, 0.0, 0.625, -1.875, 0.0, -1.875]), tol=1e-15)
