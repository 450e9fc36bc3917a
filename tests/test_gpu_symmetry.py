"""Triangle storage of K (pms_elements_set_symmetry): the CSR values hold the lower (column <= row,
russell_sparse Sym::YesLower) or upper (column >= row, Sym::YesUpper) triangle, as LinearSystem::new
picks it from the linear solver (src/fem/linear_system.rs:96-119) and assemble_matrix keeps the
entries (src/base/assembly.rs:92-122).

Each kept entry must carry the bits of the same entry of the full matrix (same summation order), on
the device-memory path, on the host-memory path (row slabs copied while later slabs gather) and in
the fused call; the full matrix itself is checked against the oracle at 1e-12."""
import numpy as np
import pytest
import torch

import oracle
from gpu_util import assert_close, perturbed_mesh, plastic_ddu
from pmsim_b200 import _lib
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu

E, NU, H, Z0 = 2e5, 0.3, 1e3, 250.0
KINDS = [M.TRI3, M.TRI6, M.QUA4, M.QUA8, M.QUA9, M.TET4, M.HEX8, M.HEX20, M.TRI15]


def _triangle(indptr, indices, values, sym):
    """The entries of a full CSR matrix that the triangle sym keeps, in row order."""
    rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    keep = indices <= rows if sym == "lower" else indices >= rows
    counts = np.add.reduceat(keep.astype(np.int64), indptr[:-1]) if len(indices) else np.zeros(0, np.int64)
    counts[np.diff(indptr) == 0] = 0
    ptr = np.concatenate([[0], np.cumsum(counts)])
    return ptr, indices[keep], values[keep]


def _elements(kind, n):
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=3, n=n)
    return m, Elements(m, Material.von_mises(E, NU, H, Z0))


@pytest.mark.parametrize("kind", KINDS, ids=[M.KIND_NAMES[k] for k in KINDS])
def test_triangles_hold_the_full_matrix_bits(kind):
    n = (6, 5, 1) if M.KIND_NDIM[kind] == 2 else (3, 3, 2)
    m, g = _elements(kind, n)
    o = oracle.OracleElements(m, 1, oracle.Params(E, NU, H, Z0), sym_tol=-1.0)
    ddu = plastic_ddu(m, seed=5)
    g.initialize_internal_values()
    g.backup_secondary_values()
    ip, ix = g.csr_pattern()
    ff, full = np.zeros(g.ndof), np.zeros(g.nnz)
    g.update_and_assemble(ddu, ff, full)
    o.initialize()
    o.update_secondary_values(ddu)
    oip, oix, ov = o.assemble_kk_csr()
    assert np.array_equal(oip, ip) and np.array_equal(oix, ix)
    assert_close(full, ov, what="K full")
    nnz_full = g.nnz
    assert g.symmetric_jacobian()  # von Mises: symmetric_stiffness() is true (von_mises.rs:92-94)
    for sym in ("lower", "upper"):
        tp, tx, tv = _triangle(ip, ix, full, sym)
        g.set_symmetry(sym)
        assert g.nnz == len(tx) and g.info.nnz == len(tx)
        # a symmetric matrix keeps its diagonal and half of the rest
        assert 2 * g.nnz - g.ndof == nnz_full
        gp, gx = g.csr_pattern()
        assert np.array_equal(gp, tp) and np.array_equal(gx, tx)
        # fused call, host memory (slab path)
        ff2, kv = np.zeros(g.ndof), np.zeros(g.nnz)
        g.update_and_assemble(ddu, ff2, kv)
        assert kv.tobytes() == tv.tobytes(), f"{sym}: fused host values"
        assert ff2.tobytes() == ff.tobytes()
        # separate call, host memory, and device memory
        assert g.assemble_kk().tobytes() == tv.tobytes(), f"{sym}: assemble_kk host values"
        dev = torch.full((g.nnz,), np.nan, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()  # the fill ran on torch's stream; the handle runs on its own
        g.assemble_kk(dev)
        g.sync()
        assert dev.cpu().numpy().tobytes() == tv.tobytes(), f"{sym}: device values"
        # the triangle against the oracle's entries (Sym::YesLower / YesUpper keep the same sums)
        assert_close(kv, _triangle(oip, oix, ov, sym)[2], what=f"K {sym}")
    g.set_symmetry("full")
    assert g.nnz == nnz_full
    assert g.assemble_kk().tobytes() == full.tobytes()


def test_triangles_at_size_hex20():
    """Many gather blocks and both row kinds of the structured block (corner, edge, face, interior)."""
    m, g = _elements(M.HEX20, (8, 6, 5))
    ddu = plastic_ddu(m, seed=9)
    g.initialize_internal_values()
    g.backup_secondary_values()
    ip, ix = g.csr_pattern()
    full = np.zeros(g.nnz)
    g.update_and_assemble(ddu, None, full)
    for sym in ("lower", "upper"):
        g.set_symmetry(sym)
        kv = np.zeros(g.nnz)
        g.update_and_assemble(ddu, None, kv)
        assert kv.tobytes() == _triangle(ip, ix, full, sym)[2].tobytes()


def test_triangles_need_the_gather_assembly():
    _, g = _elements(M.QUA8, (4, 3, 1))
    g.set_symmetry("lower")
    with pytest.raises(_lib.PmsError) as e:
        g.set_assembly("direct")
    assert e.value.code == _lib.PMS_ERR_UNSUPPORTED
    g.set_symmetry("full")
    g.set_assembly("direct")
    with pytest.raises(_lib.PmsError) as e:
        g.set_symmetry("upper")
    assert e.value.code == _lib.PMS_ERR_UNSUPPORTED
