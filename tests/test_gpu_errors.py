"""Error paths of the element calls and the batched solver, on host-made inputs, against the oracle.

The reference stops at the first error of its loops (src/fem/elements.rs:156-181): every cell's
stress update before any tangent, cells and IPs in ascending order.  The device reports the same
error, cell and IP: zero sigma_d in the update (src/material/von_mises.rs:212-216), zero norm_s in the
tangent (von_mises.rs:147-150), both when they meet (the update error wins), a refused yield-surface
size (von_mises.rs:68-70), NaN propagating through the element path without an element error (the
Newton loop then stops with "Found NaN or Inf", src/fem/convergence_control.rs:60,80-84), and, in a
batch, failing problems that stop alone while every other problem keeps its bits.
"""
import math

import numpy as np
import pytest

import error_cases as C
import oracle
from oracle.driver import OracleSolver
from pmsim_b200 import _lib
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu

ZERO_SIGMA_D = "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)"
ZERO_NORM_S = "von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)"


def handles(kind):
    from pmsim_b200.elements import Elements, Material
    m = C.shear_mesh(kind)
    g = Elements(m, Material.von_mises(C.E, C.NU, C.H_SOFT, C.Z0))
    o = oracle.OracleElements(m, oracle.MODEL_VON_MISES, oracle.Params(C.E, C.NU, C.H_SOFT, C.Z0), sym_tol=-1.0)
    g.initialize_internal_values()
    o.initialize()
    return m, g, o


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX8, M.HEX20], ids=["qua8", "hex8", "hex20"])
def test_zero_sigma_d_reports_the_references_cell_and_ip(kind):
    m, g, o = handles(kind)
    ddu = C.band_shear(m, [(4.0, 8.0, C.GAMMA_ZERO_SIGMA_D)])
    with pytest.raises(oracle.OracleError) as ref:
        o.update_secondary_values(ddu)
    with pytest.raises(_lib.PmsError) as dev:
        g.update_secondary_values(ddu)
    assert dev.value.code == _lib.PMS_ERR_ZERO_SIGMA_D and str(dev.value) == ZERO_SIGMA_D
    assert g.error_location() == (ref.value.cell, ref.value.ip) == (C.cells_inside(m, 4.0, 8.0)[0], 0)


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX8], ids=["qua8", "hex8"])
def test_zero_norm_s_in_the_tangent(kind):
    m, g, o = handles(kind)
    ddu = C.band_shear(m, [(4.0, 8.0, C.GAMMA_ZERO_NORM_S)])
    o.update_secondary_values(ddu)
    g.update_secondary_values(ddu)  # the update itself passes (sigma_d = 1.1e-10 >= 1e-10)
    sig, ivs, el = g.get_state()
    assert np.array_equal(el, o.elastic)
    with pytest.raises(oracle.OracleError) as ref:
        o.assemble_kk_coo()
    with pytest.raises(_lib.PmsError) as dev:
        g.assemble_kk()
    assert dev.value.code == _lib.PMS_ERR_ZERO_NORM_S and str(dev.value) == ZERO_NORM_S
    cell, ip = g.error_location()
    assert cell == ref.value.cell == C.cells_inside(m, 4.0, 8.0)[0] and ip == 0


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX8], ids=["qua8", "hex8"])
def test_update_error_is_reported_before_a_tangent_error_of_a_lower_cell(kind):
    """Fused call: cells of the low-x band fail in the tangent, cells of the high-x band in the
    update; the reference finishes every update before any tangent, so the update error of the
    high band is the one reported."""
    m, g, o = handles(kind)
    ddu = C.band_shear(m, [(1.0, 3.0, C.GAMMA_ZERO_NORM_S), (5.0, 8.0, C.GAMMA_ZERO_SIGMA_D)])
    g.backup_secondary_values()
    with pytest.raises(oracle.OracleError) as ref:
        o.update_secondary_values(ddu)
    with pytest.raises(_lib.PmsError) as dev:
        g.update_and_assemble(ddu, np.zeros(g.ndof), np.zeros(g.nnz))
    assert dev.value.code == _lib.PMS_ERR_ZERO_SIGMA_D
    assert C.cells_inside(m, 1.0, 3.0)[0] < C.cells_inside(m, 5.0, 8.0)[0]
    assert g.error_location() == (ref.value.cell, ref.value.ip) == (C.cells_inside(m, 5.0, 8.0)[0], 0)


def test_yield_surface_size_at_or_below_1e_6_is_refused():
    from pmsim_b200.elements import Elements, Material
    m = C.shear_mesh(M.QUA8)
    for z in (1e-6, 0.0):
        with pytest.raises(_lib.PmsError) as e:
            Elements(m, Material.von_mises(C.E, C.NU, 0.0, z))
        assert e.value.code == _lib.PMS_ERR_INVALID
        assert str(e.value) == "von Mises initial size of the yield surface must > 1e-6"
    Elements(m, Material.von_mises(C.E, C.NU, 0.0, 1.01e-6)).close()


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX20], ids=["qua8", "hex20"])
def test_nan_in_ddu_propagates_without_an_element_error(kind):
    """As in the reference, NaN reaches the IP state and F_int with no error from the element path."""
    from gpu_util import plastic_ddu, perturbed_mesh
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=2, n=(4, 3, 1) if M.KIND_NDIM[kind] == 2 else (2, 2, 2))
    ddu = plastic_ddu(m, seed=1)
    ddu[m.ndim * int(m.cells[1, 0])] = np.nan
    g = Elements(m, Material.von_mises(2e5, 0.3, 1e3, 250.0))
    o = oracle.OracleElements(m, 1, oracle.Params(2e5, 0.3, 1e3, 250.0), sym_tol=-1.0)
    g.initialize_internal_values()
    o.initialize()
    g.update_secondary_values(ddu)  # no exception
    o.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    assert np.array_equal(np.isnan(sig), np.isnan(o.sig)) and np.isnan(sig).any()
    ok = ~np.isnan(o.sig)
    assert np.max(np.abs(sig[ok] - o.sig[ok])) <= 1e-12 * np.max(np.abs(o.sig[ok]))
    ff = g.assemble_f_int()
    fo = o.assemble_f_int()
    assert np.array_equal(np.isnan(ff), np.isnan(fo)) and np.isnan(ff).any()


def _footing(nx, ny, E, z0, width, nsteps, nan_from=None):
    """Footing of the batched configuration; nan_from: the prescribed indentation is NaN from that
    load time on (a host-made NaN in the Newton loop)."""
    from test_gpu_batch import footing
    p = footing(nx, ny, E, z0, width, nsteps=nsteps)
    if nan_from is not None:
        fn = (lambda t, t0=nan_from: math.nan if t >= t0 else t)
        p.essential = [(eq, c, fn if f is not None else None) for eq, c, f in p.essential]
    return p


def _oracle_failure(p):
    """(load step index, message) at which the oracle driver stops on problem p, or None."""
    mt = p.material
    done = []
    try:
        oel = oracle.OracleElements(p.mesh, 1, oracle.Params(mt.young, mt.poisson, mt.hh, mt.z_ini), ngauss=9,
                                    sym_tol=-1.0)
        OracleSolver(oel, p.mesh.ndof, p.essential, n_max_iterations=20, t_fin=float(p.nsteps)).solve(
            lambda step, t, u, el: done.append(step))
    except Exception as e:  # the reference's error text
        msg = str(e)
        if isinstance(e, oracle.OracleError) and e.code == 4:
            msg = "the determinant of the Jacobian must be positive"
        return len(done), msg
    return None


def test_failing_problems_stop_alone_and_leave_the_others_bits():
    """Two problems fail in one batch -- a NaN prescribed value from the second load step and a cell
    with reflected node order (negative Jacobian) -- each at the step and with the message the oracle
    driver gives; the other problems' U, IP state and iteration counts are bit-identical to a batch
    without the failing ones."""
    from pmsim_b200.batch import BatchSolver
    good = [_footing(6, 3, 1e4, 9.0, 1.0, 3), _footing(5, 4, 1.5e4, 12.0, 1.5, 3), _footing(7, 3, 8e3, 7.0, 0.8, 3)]
    bad_nan = _footing(6, 3, 1e4, 9.0, 1.0, 3, nan_from=2.0)
    bad_jac = _footing(6, 3, 1e4, 9.0, 1.0, 3)
    bad_jac.mesh = C.inverted(bad_jac.mesh, 7)
    mix = [good[0], bad_nan, good[1], bad_jac, good[2]]
    for on_fail_mode in ("lock_step", "independent"):
        a = BatchSolver(mix, n_max_iterations=20)
        if on_fail_mode == "lock_step":
            a.solve(on_fail="drop")
        else:
            a.solve_independent(on_fail="drop")
        assert set(a.failed) == {1, 3}
        for i, p in ((1, bad_nan), (3, bad_jac)):
            ref = _oracle_failure(p)
            assert ref is not None and a.failed[i] == ref, (i, a.failed[i], ref)
        b = BatchSolver(good, n_max_iterations=20)
        if on_fail_mode == "lock_step":
            b.solve(on_fail="raise")
        else:
            b.solve_independent(on_fail="raise")
        ua, ub = a.u(), b.u()
        sa, sb = a.elements.get_state(), b.elements.get_state()
        for j, i in enumerate((0, 2, 4)):
            assert np.array_equal(a.u_of(i, ua), b.u_of(j, ub)), f"problem {i}: U differs"
            for x, y in zip(a.state_of(i, sa), b.state_of(j, sb)):
                assert np.array_equal(x, y), f"problem {i}: IP state differs"
            assert a.history[i] == b.history[j]
        a.close()
        b.close()


DIVERGENCE = {"Newton-Raphson did not converge",
              "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)"}


def _dropin_failure(p):
    """(load step index, message) at which the drop-in path (device elements, host direct solve, the
    reference's Newton loop) stops on problem p, or None."""
    from pmsim_b200.elements import Elements
    from pmsim_b200.solver import SolverImplicit
    el = Elements(p.mesh, p.material, ngauss=9)
    done = []
    try:
        SolverImplicit(el, p.essential, n_max_iterations=20, t_fin=float(p.nsteps)).solve(
            lambda step, t, u, e: done.append(step))
    except Exception as e:  # the reference's error text
        return len(done), str(e)
    finally:
        el.close()
    return None


def test_population_sample_fails_where_the_oracle_driver_fails():
    """A seeded sample of 32 footings from the batched configuration's population (512, seed 2024).
    * The batched device solver, as the benchmark runs it (independent progress, failing problems
      dropped), stops exactly the problems the oracle driver (direct solve) stops, at the same load
      step.  Its linear solves are PCG to 1e-12 relative, so inside a diverging step its iterates
      are not the direct solve's: a diverging Newton loop on this perfectly plastic material either
      drives some sigma_d to zero or runs out of iterations, and which shows first may differ.  The
      message must match, or both must be one of those two.
    * The drop-in path (device elements with the same direct solve as the oracle) stops every
      problem that fails on either side at the oracle's step with the oracle's message."""
    from pmsim_b200.batch import BatchSolver
    from pmsim_b200.footing import population
    probs = population(512, seed=2024)
    rng = np.random.default_rng(11)
    sample = sorted(rng.choice(512, size=32, replace=False).tolist())
    bs = BatchSolver([probs[i] for i in sample], n_max_iterations=20, pcg_max_iterations=5000)
    bs.solve_independent(on_fail="drop")
    bad = []
    nfail = 0
    for k, i in enumerate(sample):
        ref = _oracle_failure(probs[i])
        got = bs.failed.get(k)
        if ref is None and got is None:
            continue
        nfail += 1
        same_step = (ref is None) == (got is None) and (ref is None or ref[0] == got[0])
        same_msg = ref is not None and got is not None and (ref[1] == got[1] or {ref[1], got[1]} <= DIVERGENCE)
        drop = _dropin_failure(probs[i])
        if not (same_step and same_msg and drop == ref):
            bad.append((i, probs[i].name, "oracle", ref, "batched", got, "drop-in", drop))
    bs.close()
    assert not bad, bad
    assert nfail > 0, "the sample holds failing problems"
