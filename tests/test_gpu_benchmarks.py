"""The reference's linear-elastic benchmark tests through the device element path, at the
reference tests' own tolerances (the oracle replays of the same problems are in
test_oracle_benchmarks.py): Felippa's thick cylinder (axisymmetric Qua8, u_r to 1e-15), Durand and
Farias' strip footing (nodal stresses against the closed form), the Newton solve with prescribed
displacements and Lagrange multipliers, and the one-element partitioned and residual approaches
built from the device's element calls."""
import numpy as np
import pytest

import problems
from test_oracle_benchmarks import check_strip_footing, prescribed_direct_approach, prescribed_residual_approach

pytestmark = pytest.mark.gpu


def _elements(pb, ngauss=0, axisymmetric=False):
    from pmsim_b200.elements import Elements, Material
    return Elements(pb["mesh"], Material.linear_elastic(pb["young"], pb["poisson"]), ngauss=ngauss,
                    axisymmetric=axisymmetric)


def _solve(pb, el, lmm):
    from pmsim_b200.solver import SolverImplicit
    out = {}
    SolverImplicit(el, pb["essential"], lagrange_mult_method=lmm, t_fin=1.0, natural=pb.get("natural")).solve(
        lambda s, t, u, e: out.setdefault("u", np.array(u[:pb["mesh"].ndof])))
    return out["u"]


def test_felippa_thick_cylinder_axisymmetric_on_device():
    pb = problems.felippa_thick_cylinder()
    el = _elements(pb, pb["ngauss"], True)
    u = _solve(pb, el, lmm=False)
    m = pb["mesh"]
    for p in pb["check_points"]:
        assert abs(u[2 * p] - pb["ur"](m.coords[p, 0])) < pb["tol"], p
    el.close()


def test_durand_farias_strip_footing_on_device():
    pb = problems.durand_farias_example4()
    el = _elements(pb, pb["ngauss"])
    _solve(pb, el, lmm=False)
    check_strip_footing(pb, el.get_state()[0])
    el.close()


def test_prescribe_displacements_2d_on_device():
    pb = problems.prescribe_displacements_2d()
    el = _elements(pb)
    u = _solve(pb, el, lmm=True)
    np.testing.assert_allclose(u[:8], pb["expected"], rtol=0, atol=pb["tol"])
    el.close()


class _DeviceCalls:
    """The reference test's element calls on the device (one cell: local = global)."""

    def __init__(self, pb):
        self.el = _elements(pb)
        self.el.initialize_internal_values()

    def update(self, ddu):
        self.el.update_secondary_values(ddu)

    def f_int(self):
        return self.el.calc_f_int(0)

    def jacobian(self):
        return self.el.calc_jacobian(0)

    def stresses(self):
        return self.el.get_state()[0]


def test_solid_prescribed_displacement_both_approaches_on_device():
    pb = problems.solid_prescribed_displacement()
    for approach in (prescribed_direct_approach, prescribed_residual_approach):
        calls = _DeviceCalls(pb)
        approach(pb, calls)
        calls.el.close()
