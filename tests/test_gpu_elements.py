"""K2 parity: fused element kernels + deterministic CSR gather vs the CPU oracle, every kind.

Reference: ElementSolid::{update_secondary_values, calc_f_int, calc_jacobian}
(src/fem/element_solid.rs:124-224), Elements loops (src/fem/elements.rs:132-205), COO assembly
(src/base/assembly.rs:38-139).  Tolerance: relative (normwise) 1e-12; CSR bit-reproducible.
"""
import numpy as np
import pytest

import oracle
from gpu_util import assert_close, perturbed_mesh, plastic_ddu
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu

E, NU, H, Z0 = 2e5, 0.3, 1e3, 250.0
KINDS = [M.TRI3, M.TRI6, M.QUA4, M.QUA8, M.QUA9, M.TET4, M.HEX8, M.HEX20, M.TRI10, M.TRI15]
GRID = {2: (4, 3, 1), 3: (2, 2, 2)}


def make(kind, model=1, ngauss=0, seed=0):
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=seed, n=GRID[M.KIND_NDIM[kind]])
    mat = Material.von_mises(E, NU, H, Z0) if model == 1 else Material.linear_elastic(E, NU)
    g = Elements(m, mat, ngauss=ngauss)
    o = oracle.OracleElements(m, model, oracle.Params(E, NU, H, Z0), ngauss=ngauss, sym_tol=-1.0)
    return m, g, o


def oracle_csr_values(o, indptr, indices):
    ip, ix, data = o.assemble_kk_csr()
    assert np.array_equal(ip, indptr) and np.array_equal(ix, indices)
    return data


@pytest.mark.parametrize("kind", KINDS, ids=[M.KIND_NAMES[k] for k in KINDS])
def test_fused_update_and_assemble_matches_oracle(kind):
    m, g, o = make(kind)
    indptr, indices = g.csr_pattern()
    g.initialize_internal_values()
    o.initialize()
    # iteration 0 of a step: assemble from the initial (elastic) state
    assert np.all(g.assemble_f_int() == 0.0)
    k0 = g.assemble_kk()
    assert_close(k0, oracle_csr_values(o, indptr, indices), what="K elastic")
    # one Newton update from the backed-up state, then F_int and K on the updated state
    ddu = plastic_ddu(m, seed=kind)
    g.backup_secondary_values()
    ff = np.zeros(g.ndof)
    kv = np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff, kv)
    o.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    assert np.array_equal(el, o.elastic), "elastic flags differ"
    assert 0 < (1 - el.mean()) < 1, "expected a mix of elastic and plastic IPs"
    assert_close(sig, o.sig, what="sigma")
    assert_close(ivs, o.ivs, what="[z, lambda]")
    assert_close(ff, o.assemble_f_int(), what="f_int")
    assert_close(kv, oracle_csr_values(o, indptr, indices), what="K")


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX20], ids=["qua8", "hex20"])
def test_separate_calls_match_fused(kind):
    """update_secondary + assemble_f_int + assemble_kk == fused call (to rounding: the two kernel
    instantiations may fuse multiply-adds differently)."""
    m, g, o = make(kind, seed=3)
    ddu = plastic_ddu(m, seed=5)
    g.initialize_internal_values()
    g.backup_secondary_values()
    ff1, kv1 = np.zeros(g.ndof), np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff1, kv1)
    s1 = g.get_state()
    g.restore_secondary_values()
    g.update_secondary_values(ddu)
    ff2 = g.assemble_f_int()
    kv2 = g.assemble_kk()
    s2 = g.get_state()
    assert_close(ff1, ff2, tol=1e-13, what="f_int")
    assert_close(kv1, kv2, tol=1e-13, what="K")
    assert_close(s1[0], s2[0], tol=1e-13, what="sigma")
    assert_close(s1[1], s2[1], tol=1e-13, what="[z, lambda]")
    assert np.array_equal(s1[2], s2[2])


@pytest.mark.parametrize("kind", [M.QUA4, M.QUA8, M.HEX8, M.HEX20], ids=["qua4", "qua8", "hex8", "hex20"])
def test_per_cell_calls_match_oracle(kind):
    m, g, o = make(kind, seed=7)
    ddu = plastic_ddu(m, seed=9)
    g.initialize_internal_values()
    g.update_secondary_values(ddu)
    o.initialize()
    o.update_secondary_values(ddu)
    ng, nc = g.ngauss, g.ncomp
    for cell in [0, m.ncell // 2, m.ncell - 1]:
        X = m.coords[m.cells[cell]]
        sl = slice(cell * ng, (cell + 1) * ng)
        kf = oracle.elem_jacobian(kind, ng, X, 1, oracle.Params(E, NU, H, Z0), o.sig[sl], o.ivs[sl], o.elastic[sl])
        assert_close(g.calc_jacobian(cell), kf, what=f"K_e cell {cell}")
        assert_close(g.calc_f_int(cell), oracle.elem_f_int(kind, ng, X, o.sig[sl]), what=f"f_e cell {cell}")


def test_csr_bit_reproducible():
    m, g, o = make(M.HEX20, seed=1)
    ddu = plastic_ddu(m, seed=2)
    g.initialize_internal_values()
    g.backup_secondary_values()
    outs = []
    for _ in range(3):
        ff, kv = np.zeros(g.ndof), np.zeros(g.nnz)
        g.update_and_assemble(ddu, ff, kv)
        outs.append((ff.tobytes(), kv.tobytes()))
    assert outs[0] == outs[1] == outs[2]


@pytest.mark.parametrize("kind", KINDS, ids=[M.KIND_NAMES[k] for k in KINDS])
def test_direct_and_gather_assembly_agree(kind):
    """The direct assembly (blocks added straight into the CSR values and R, every entry summed over
    its cells in the colour-major processing order) gives the same bits on every run, and agrees with
    the gather assembly (upper element-matrix blocks, then row gathers in ascending cell order) to
    1e-13: the summation orders differ and the two are different kernel instantiations, which the
    compiler may contract into fused multiply-adds differently, so only the last bits may differ (a
    missing or doubled block would differ at O(1))."""
    m, g, o = make(kind, seed=7)
    ddu = plastic_ddu(m, seed=8)
    g.initialize_internal_values()
    g.backup_secondary_values()
    got = {}
    for mode in ("direct", "gather", "direct"):
        g.set_assembly(mode)
        ff, kv = np.zeros(g.ndof), np.zeros(g.nnz)
        g.update_and_assemble(ddu, ff, kv)
        f2 = g.assemble_f_int()
        k2 = g.assemble_kk()
        got.setdefault(mode, []).append((ff, kv, f2, k2))
    d0, d1, ga = got["direct"][0], got["direct"][1], got["gather"][0]
    for a, b in zip(d0, d1):
        assert a.tobytes() == b.tobytes(), "direct assembly not reproducible"
    for a, b, what in zip(d0, ga, ("f_int", "K", "f_int (separate)", "K (separate)")):
        assert_close(a, b, tol=1e-13, what=what)
    assert 0 < 1 - g.get_state()[2].mean() < 1


@pytest.mark.parametrize("ngauss", [4, 9])
def test_qua8_gauss_rules(ngauss):
    m, g, o = make(M.QUA8, ngauss=ngauss, seed=4)
    ddu = plastic_ddu(m, seed=4)
    g.initialize_internal_values()
    g.update_secondary_values(ddu)
    o.initialize()
    o.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    assert_close(sig, o.sig, what="sigma")
    assert_close(g.assemble_kk(), oracle_csr_values(o, *g.csr_pattern()), what="K")


def test_linear_elastic_and_materials_per_cell():
    """cell_material selects the parameters per cell (cell attribute -> ParamSolid)."""
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(M.QUA8, seed=8, n=(4, 2, 1))
    cm = (np.arange(m.ncell) % 2).astype(np.int32)
    mats = [Material.von_mises(E, NU, H, Z0), Material.linear_elastic(2 * E, 0.25)]
    g = Elements(m, mats, cell_material=cm)
    ddu = plastic_ddu(m, seed=8)
    g.initialize_internal_values()
    g.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    ng = g.ngauss
    for c in range(m.ncell):
        model = 1 if cm[c] == 0 else 0
        prm = oracle.Params(E, NU, H, Z0) if model == 1 else oracle.Params(2 * E, 0.25)
        sub = oracle.OracleElements(M.Mesh(2, m.coords, m.cells[c:c + 1], M.QUA8), model, prm)
        sub.initialize()
        sub.update_secondary_values(ddu)
        assert_close(sig[c * ng:(c + 1) * ng], sub.sig, what=f"cell {c}")


def test_errors_are_reported_with_location():
    """A collapsed cell gives the Jacobian error with its cell id (no GPU fault)."""
    from pmsim_b200.elements import Elements, Material
    from pmsim_b200._lib import PmsError
    m = M.structured_2d(M.QUA4, 2, 1, 2.0, 1.0)
    c = m.coords.copy()
    c[m.cells[1][2]] = c[m.cells[1][0]]  # fold cell 1
    g = Elements(M.Mesh(2, c, m.cells, M.QUA4), Material.von_mises(E, NU, H, Z0))
    with pytest.raises(PmsError) as ei:
        g.assemble_kk()
    assert "Jacobian" in str(ei.value)
    assert g.error_location()[0] == 1


def test_femstate_checkpoint_round_trip_on_device():
    """Export the device IP state in pmsim's FemState JSON layout and import it into a fresh handle."""
    from pmsim_b200 import state_io
    m, g, o = make(M.QUA8, seed=12)
    ddu = plastic_ddu(m, seed=12)
    g.initialize_internal_values()
    g.update_secondary_values(ddu)
    text = state_io.export_state(g, u=ddu, ddu=ddu, t=1.0)
    from pmsim_b200.elements import Elements, Material
    h = Elements(m, Material.von_mises(E, NU, H, Z0))
    u, du, t = state_io.import_state(h, text)
    assert t == 1.0 and np.array_equal(u, ddu)
    for a, b in zip(g.get_state(), h.get_state()):
        assert np.array_equal(a, b)
    assert state_io.export_state(h, u=u, ddu=du, t=t) == text


KINDS_2D = [M.TRI3, M.TRI6, M.QUA4, M.QUA8, M.QUA9]


@pytest.mark.parametrize("kind", KINDS_2D, ids=[M.KIND_NAMES[k] for k in KINDS_2D])
def test_axisymmetric_update_and_assemble_matches_oracle(kind):
    """Axisymmetric idealization (x = radius): weight |J| w r, hoop strain u_r/r, hoop rows of B in
    F_int and K (src/base/calculate_strain.rs:36-48, gemlab integrators with args.axisymmetric,
    src/fem/element_solid.rs:128-171), von Mises with plastic and elastic IPs, against the oracle."""
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=7, n=GRID[2])
    m.coords[:, 0] += 0.5  # keep every point off the axis
    g = Elements(m, Material.von_mises(E, NU, H, Z0), axisymmetric=True)
    o = oracle.OracleElements(m, 1, oracle.Params(E, NU, H, Z0), sym_tol=-1.0, axisymmetric=True)
    indptr, indices = g.csr_pattern()
    g.initialize_internal_values()
    o.initialize()
    assert_close(g.assemble_kk(), oracle_csr_values(o, indptr, indices), what="K elastic")
    ddu = plastic_ddu(m, seed=kind + 40)
    g.backup_secondary_values()
    ff = np.zeros(g.ndof)
    kv = np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff, kv)
    o.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    assert np.array_equal(el, o.elastic), "elastic flags differ"
    assert 0 < (1 - el.mean()) < 1, "expected a mix of elastic and plastic IPs"
    assert_close(sig, o.sig, what="sigma")
    assert_close(ivs, o.ivs, what="[z, lambda]")
    assert_close(ff, o.assemble_f_int(), what="f_int")
    assert_close(kv, oracle_csr_values(o, indptr, indices), what="K")


def test_sgm_5d17_axisymmetric_on_device():
    """tests/test_solid_smith_5d17_qua4_axisym.rs on the device elements (two layers, 9 IP, point
    loads, reduced-system method): the reference test's displacements at its tolerance 1e-9."""
    import problems
    from pmsim_b200.elements import Elements, Material
    from pmsim_b200.solver import SolverImplicit
    pb = problems.sgm_5d17_axisym()
    mats = [Material.linear_elastic(E_, nu) for E_, nu in pb["mats"]]
    el = Elements(pb["mesh"], mats, ngauss=9, cell_material=pb["cmat"], axisymmetric=True)
    sol = SolverImplicit(el, pb["essential"], loads=pb["loads"], lagrange_mult_method=False, t_fin=1.0)
    out = {}
    sol.solve(lambda step, t, u, e: out.setdefault("u", u.copy()))
    np.testing.assert_allclose(out["u"], pb["golden"]["uu_correct"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("kind", KINDS_2D, ids=[M.KIND_NAMES[k] for k in KINDS_2D])
def test_plane_stress_update_and_assemble_matches_oracle(kind):
    """Plane stress (linear elastic; in-plane normal block E/(1-nu^2) (1, nu; nu, 1), no sigma_zz) with
    thickness 0.25, against the oracle."""
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=9, n=GRID[2])
    g = Elements(m, Material.linear_elastic(E, NU), thickness=0.25, plane_stress=True)
    o = oracle.OracleElements(m, oracle.MODEL_LINEAR_ELASTIC_PLANE_STRESS, oracle.Params(E, NU, 0.0, 1.0), thickness=0.25)
    indptr, indices = g.csr_pattern()
    g.initialize_internal_values()
    o.initialize()
    ddu = plastic_ddu(m, seed=kind + 60)
    g.backup_secondary_values()
    ff = np.zeros(g.ndof)
    kv = np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff, kv)
    o.update_secondary_values(ddu)
    sig = g.get_state()[0]
    assert np.all(sig[:, 2] == 0.0), "plane stress keeps sigma_zz = 0"
    assert_close(sig, o.sig, what="sigma")
    assert_close(ff, o.assemble_f_int(), what="f_int")
    assert_close(kv, oracle_csr_values(o, indptr, indices), what="K")


def test_bhatti_1d6_plane_stress_on_device():
    """tests/test_solid_bhatti_1d6_plane_stress.rs on the device elements: the reference test's
    displacements (its tolerance is 1e-15; the device sums in another order, so 1e-14 here)."""
    import problems
    from pmsim_b200.elements import Elements, Material
    from pmsim_b200.solver import SolverImplicit
    pb = problems.bhatti_1d6_plane_stress()
    el = Elements(pb["mesh"], Material.linear_elastic(pb["young"], pb["poisson"]), thickness=pb["thickness"],
                  plane_stress=True)
    sol = SolverImplicit(el, pb["essential"], lagrange_mult_method=False, t_fin=1.0, natural=pb["natural"])
    out = {}
    sol.solve(lambda step, t, u, e: out.setdefault("u", u.copy()))
    np.testing.assert_allclose(out["u"], pb["golden"]["uu_correct"], rtol=0, atol=1e-14)
