"""GPU parity at the sizes of the benchmark configurations (or large enough to take the same code
paths), against the CPU oracle.

* Hex20 24x24x12 (6,912 cells): the persistent element kernel walks its cell list in about six waves
  of resident blocks and the CSR assembly spans thousands of blocks.
* Qua8 128x63 (8,064 cells, a number not divisible by three): the packed 2D kernel with a ragged
  last group of three 10-lane cells, over many blocks.
* The 20x10 Qua8 strip footing exactly as configured (9 IP, 10 load steps): the drop-in path
  (device elements + host direct solve) and the batched device solver, against the oracle's Newton
  loop, at every step.
* The von Mises batch kernel on 1,048,576 IPs drawn as the 16.8M-IP microbenchmark draws them.

Reference: ElementSolid::{update_secondary_values, calc_f_int, calc_jacobian}
(src/fem/element_solid.rs:124-224), assembly (src/base/assembly.rs:38-139), SolverImplicit::iterate
(src/fem/solver_implicit.rs:187-272), VonMises (src/material/von_mises.rs:124-226).
"""
import numpy as np
import pytest

import oracle
from gpu_util import TOL, assert_close, perturbed_mesh, plastic_ddu
from oracle.driver import OracleSolver
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu


def fused_vs_oracle(m, mat_args, ngauss, ddu):
    from pmsim_b200.elements import Elements, Material
    g = Elements(m, Material.von_mises(*mat_args), ngauss=ngauss)
    o = oracle.OracleElements(m, 1, oracle.Params(*mat_args), ngauss=ngauss, sym_tol=-1.0, nthreads=0)
    g.initialize_internal_values()
    o.initialize()
    g.backup_secondary_values()
    ff, kv = np.zeros(g.ndof), np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff, kv)
    o.update_secondary_values(ddu)
    sig, ivs, el = g.get_state()
    assert np.array_equal(el, o.elastic), "elastic flags differ"
    frac = 1.0 - el.mean()
    assert 0.05 < frac < 0.95, frac
    assert_close(sig, o.sig, what="sigma")
    assert_close(ivs, o.ivs, what="[z, lambda]")
    assert_close(ff, o.assemble_f_int(), what="f_int")
    indptr, indices = g.csr_pattern()
    ip, ix, data = o.assemble_kk_csr()
    assert np.array_equal(ip, indptr) and np.array_equal(ix, indices)
    assert_close(kv, data, what="K")
    kv2 = np.zeros(g.nnz)
    g.update_and_assemble(ddu, None, kv2)
    assert np.array_equal(kv, kv2), "CSR values differ between two runs"
    # the other assembly (direct: blocks added straight into the CSR values) at the same size
    g.set_assembly("direct")
    ff3, kv3 = np.zeros(g.ndof), np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff3, kv3)
    assert_close(ff3, o.assemble_f_int(), what="f_int (direct)")
    assert_close(kv3, data, what="K (direct)")
    kv4 = np.zeros(g.nnz)
    g.update_and_assemble(ddu, None, kv4)
    assert np.array_equal(kv3, kv4), "direct CSR values differ between two runs"
    g.close()


def test_hex20_block_several_waves():
    m = perturbed_mesh(M.HEX20, seed=4, n=(24, 24, 12), amp=0.05)
    fused_vs_oracle(m, (2e5, 0.3, 1e3, 250.0), 0, plastic_ddu(m, seed=9, strain=6e-4))  # about half plastic


def test_qua8_ragged_groups():
    m = perturbed_mesh(M.QUA8, seed=4, n=(128, 63, 1), amp=0.05)
    fused_vs_oracle(m, (1e4, 0.3, 0.0, 9.0), 9, plastic_ddu(m, seed=9, strain=3e-4))  # about half plastic


def _c0():
    from pmsim_b200.footing import footing_problem
    return footing_problem(20, 10, 1e4, 9.0, 1.0, nsteps=10)


def _oracle_c0(p):
    mt = p.material
    oel = oracle.OracleElements(p.mesh, 1, oracle.Params(mt.young, mt.poisson, mt.hh, mt.z_ini), ngauss=9,
                                sym_tol=-1.0)
    ref = []
    osol = OracleSolver(oel, p.mesh.ndof, p.essential, n_max_iterations=20, t_fin=10.0)
    osol.solve(lambda step, t, u, el: ref.append((u.copy(), el.sig.copy())))
    return ref, [len(h) for h in osol.history]


def test_c0_footing_dropin_path_matches_oracle_every_step():
    """Drop-in path: the device computes every element call, SuperLU solves (as the oracle does)."""
    from pmsim_b200.elements import Elements
    from pmsim_b200.solver import SolverImplicit
    p = _c0()
    ref, ref_iters = _oracle_c0(p)
    el = Elements(p.mesh, p.material, ngauss=9)
    got = []
    sol = SolverImplicit(el, p.essential, n_max_iterations=20, t_fin=10.0)
    sol.solve(on_step=lambda k, t, u, e: got.append((u.copy(), e.get_state()[0])))
    assert [len(h) for h in sol.history] == ref_iters == [7, 7, 6, 6, 6, 7, 7, 5, 5, 5]
    assert len(got) == len(ref) == 10
    # same element arithmetic (1e-12) and the same direct solver: the iterates agree to rounding
    for k, ((ug, sg), (uo, so)) in enumerate(zip(got, ref)):
        assert_close(ug, uo, tol=1e-11, what=f"step {k} U")
        assert_close(sg, so, tol=1e-10, what=f"step {k} sigma")
    el.close()


def test_c0_footing_batched_solver_matches_oracle_every_step():
    """Batched device solver: FP64 block-Jacobi PCG to |r| <= 1e-12 |r0| in place of the direct
    solve.  Both Newton loops stop at max|R| < 1e-10 or rel(mdu) < 1e-8, so the converged U of
    each step agree to the stopping tests, not to rounding: with the footing's stiffness the
    measured gap is a few 1e-11 of max|U|; the stresses of this perfectly plastic material
    (H = 0) follow U through the return map, measured within a few 1e-9 of max|sigma|.  The
    asserted bounds leave a 10x margin over those measurements."""
    from pmsim_b200.batch import BatchSolver
    p = _c0()
    ref, ref_iters = _oracle_c0(p)
    bs = BatchSolver([p], n_max_iterations=20)
    got = []
    bs.solve(lambda s, b: got.append((b.u_of(0).copy(), b.state_of(0)[0].copy())))
    assert bs.history[0] == ref_iters
    for k, ((ug, sg), (uo, so)) in enumerate(zip(got, ref)):
        assert_close(ug, uo, tol=1e-9, what=f"step {k} U")
        assert_close(sg, so, tol=1e-7, what=f"step {k} sigma")
    bs.close()


def test_k1_on_the_microbenchmark_distribution():
    """1,048,576 IPs drawn as the 16,777,216-IP microbenchmark: sigma0 = 0, z0 = 250,
    deps ~ N(0, (1.5 z0 / 2G)^2) i.i.d. per Mandel component, H ~ U[0, 2e3], E = 2e5, nu = 0.3."""
    import torch
    from pmsim_b200.material import VonMisesBatch, unpack_tangent
    E, NU, Z0 = 2e5, 0.3, 250.0
    n = 1 << 20
    gg = E / (2 * (1 + NU))
    rng = np.random.default_rng(1234)
    deps = rng.normal(0.0, 1.5 * Z0 / (2 * gg), size=(n, 6))
    hh = rng.uniform(0.0, 2e3, n)
    o_sig = np.zeros((n, 6))
    o_ivs = np.stack([np.full(n, Z0), np.zeros(n)], 1).copy()
    o_el = np.ones(n, np.uint8)
    o_dd = oracle.model_batch_hh(1, oracle.Params(E, NU, 0.0, Z0), 3, hh, o_sig, o_ivs, o_el, deps)
    dev = torch.device("cuda:0")
    g_sig = torch.zeros((6, n), dtype=torch.float64, device=dev)
    g_z = torch.full((n,), Z0, dtype=torch.float64, device=dev)
    g_lam = torch.zeros(n, dtype=torch.float64, device=dev)
    g_el = torch.zeros(n, dtype=torch.uint8, device=dev)
    g_dd = torch.zeros((21, n), dtype=torch.float64, device=dev)
    status = torch.zeros(4, dtype=torch.int32, device=dev)
    vm = VonMisesBatch(E, NU, 0.0, Z0, ndim=3)
    vm.update_and_stiffness(g_sig, g_z, g_lam, g_el, torch.tensor(deps.T.copy(), device=dev),
                            hh=torch.tensor(hh, device=dev), dd=g_dd, status=status)
    torch.cuda.synchronize()
    assert int(status[0]) == 0
    assert np.array_equal(g_el.cpu().numpy(), o_el)
    assert 0.05 < 1.0 - o_el.mean() < 1.0
    assert_close(g_sig.cpu().numpy().T, o_sig, tol=TOL, what="sigma")
    assert_close(g_z.cpu().numpy(), o_ivs[:, 0], what="z")
    assert_close(g_lam.cpu().numpy(), o_ivs[:, 1], what="lambda")
    got = unpack_tangent(g_dd.cpu().numpy(), 6)
    # per-IP relative check of the tangent (each IP's own scale)
    scale = np.abs(o_dd).reshape(n, -1).max(1)
    err = np.abs(got - o_dd).reshape(n, -1).max(1)
    assert np.all(err <= TOL * scale), float((err / scale).max())
