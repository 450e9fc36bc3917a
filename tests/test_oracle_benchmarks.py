"""The reference's linear-elastic benchmark tests replayed by the oracle, at the reference tests'
own tolerances: Felippa's thick cylinder (axisymmetric Qua8), Durand and Farias' strip footing
(Qua4, nodal stress recovery against the closed form), and the two one-Qua4 prescribed-displacement
tests (a Newton solve with Lagrange multipliers; the partitioned and the residual approaches built
from element calls).  These pin the oracle that the device replays in test_gpu_benchmarks.py are
checked beside."""
import numpy as np

import oracle
import problems
from oracle.driver import OracleSolver


def _elements(pb, ngauss=0, axisymmetric=False):
    return oracle.OracleElements(pb["mesh"], 0, oracle.Params(pb["young"], pb["poisson"], 0.0, 1.0), ngauss=ngauss,
                                 sym_tol=-1.0, axisymmetric=axisymmetric)


def _solve(pb, el, lmm):
    out = {}
    m = pb["mesh"]
    nat = pb.get("natural")
    OracleSolver(el, m.ndof, pb["essential"], lagrange_mult_method=lmm, t_fin=1.0,
                 ff_ext_fn=nat.ff_ext if nat is not None else None).solve(
        lambda s, t, u, e: out.setdefault("u", np.array(u[:m.ndof])))
    return out["u"]


def test_oracle_felippa_thick_cylinder_axisymmetric():
    pb = problems.felippa_thick_cylinder()
    u = _solve(pb, _elements(pb, pb["ngauss"], True), lmm=False)
    m = pb["mesh"]
    for p in pb["check_points"]:
        assert abs(u[2 * p] - pb["ur"](m.coords[p, 0])) < pb["tol"], p


def test_oracle_durand_farias_strip_footing():
    pb = problems.durand_farias_example4()
    el = _elements(pb, pb["ngauss"])
    _solve(pb, el, lmm=False)
    check_strip_footing(pb, np.array(el.sig))


def check_strip_footing(pb, sig):
    m = pb["mesh"]
    c0 = m.cells[pb["left_cells"][0]]
    hdx = (m.coords[c0, 0].max() - m.coords[c0, 0].min()) / 2.0
    nodal = problems.nodal_stresses(m, pb["left_cells"], sig, pb["ngauss"], lambda x, y: x < hdx)
    assert len(nodal) == 8  # the nodes of the left edge
    for x, y, sxx, syy, sxy in nodal:
        ana = problems.strip_load_stress(x, y, pb["bb"], pb["hh"], pb["qn"], pb["poisson"])
        for v, a, tol in zip((sxx, syy, sxy), ana, pb["tols"]):
            assert abs(v - a) / pb["qn"] <= tol, (x, y, v, a)


def test_oracle_prescribe_displacements_2d():
    pb = problems.prescribe_displacements_2d()
    u = _solve(pb, _elements(pb), lmm=True)
    np.testing.assert_allclose(u[:8], pb["expected"], rtol=0, atol=pb["tol"])


class _OracleCalls:
    """The element calls the reference test makes on its one element (global = local)."""

    def __init__(self, pb):
        self.el = _elements(pb)
        self.el.initialize()

    def update(self, ddu):
        self.el.update_secondary_values(ddu)

    def f_int(self):
        return np.array(self.el.assemble_f_int())

    def jacobian(self):
        indptr, indices, vals = self.el.assemble_kk_csr()
        k = np.zeros((8, 8))
        for r in range(8):
            k[r, indices[indptr[r]:indptr[r + 1]]] = vals[indptr[r]:indptr[r + 1]]
        return k

    def stresses(self):
        return np.array(self.el.sig)


def prescribed_direct_approach(pb, calls):
    """tests/test_solid_prescribed_displacement.rs, direct approach: K11 U1 = -K12 U2, then the
    stresses and the reactions K21 U1 + K22 U2 against F_int on the prescribed equations."""
    eqp = sorted(pb["prescribed"])
    equ = pb["unknown"]
    u = np.zeros(8)
    ddu = np.zeros(8)
    for eq, v in pb["prescribed"].items():
        ddu[eq] = v - u[eq]
        u[eq] = v
    k = calls.jacobian()
    u2 = u[eqp]
    u1 = np.linalg.solve(k[np.ix_(equ, equ)], -k[np.ix_(equ, eqp)] @ u2)
    u[equ] = u1
    ddu[equ] = u1
    calls.update(ddu)
    for s in calls.stresses():
        np.testing.assert_allclose(s, pb["stress"], rtol=0, atol=pb["tol"])
    e2 = k[np.ix_(eqp, equ)] @ u1 + k[np.ix_(eqp, eqp)] @ u2
    np.testing.assert_allclose(calls.f_int()[eqp], e2, rtol=0, atol=pb["tol"])


def prescribed_residual_approach(pb, calls):
    """The same test's residual approach: update with the prescribed increments, R = F_int with the
    prescribed rows removed, K with the prescribed rows and columns replaced by unit diagonal rows,
    U -= K^-1 R, then a second update from the unknown increments only."""
    eqp = sorted(pb["prescribed"])
    equ = pb["unknown"]
    u = np.zeros(8)
    ddu = np.zeros(8)
    for eq, v in pb["prescribed"].items():
        ddu[eq] = v - u[eq]
        u[eq] = v
    calls.update(ddu)
    rr = calls.f_int()
    assert [f"{v:.6f}" for v in -rr[equ]] == [f"{v:.6f}" for v in pb["e1"]]
    rr[eqp] = 0.0
    k = calls.jacobian()
    k[eqp, :] = 0.0
    k[:, eqp] = 0.0
    k[eqp, eqp] = 1.0
    mdu = np.linalg.solve(k, rr)
    u -= mdu
    ddu -= mdu
    np.testing.assert_allclose(ddu, pb["ddu"], rtol=0, atol=pb["tol"])
    ddu[eqp] = 0.0
    calls.update(ddu)
    for s in calls.stresses():
        np.testing.assert_allclose(s, pb["stress"], rtol=0, atol=pb["tol"])


def test_oracle_solid_prescribed_displacement_both_approaches():
    pb = problems.solid_prescribed_displacement()
    prescribed_direct_approach(pb, _OracleCalls(pb))
    prescribed_residual_approach(pb, _OracleCalls(pb))
