"""The maps of the direct assembly (host only): replaying the device's order -- cells in ascending
order, each block stored by the lowest cell that holds both of its nodes and added to by the later
ones, at the slots of the maps -- with the oracle's element matrices gives the oracle's CSR values
bit for bit (the oracle sums the reference's COO duplicates in insertion order, i.e. by ascending
cell).  Also checks the ranks (ascending cell order per node, last flag) that order the row slabs."""
import ctypes

import numpy as np
import pytest

import oracle
from gpu_util import perturbed_mesh, plastic_ddu
from pmsim_b200 import _lib
from pmsim_b200 import mesh as M

CRANK_LAST = 1 << 30


def maps(m):
    L = _lib.load()
    nn = m.nnode
    cslot = np.zeros(m.ncell * nn * nn, np.int16)
    crank = np.zeros(m.ncell * nn, np.int32)
    cfirst = np.zeros(m.ncell * nn, np.uint32)
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    assert L.pms_mesh_assembly_maps(ctypes.byref(cm), _lib.ptr(cslot), _lib.ptr(crank), _lib.ptr(cfirst)) == 0
    return cslot.reshape(m.ncell, nn, nn), crank.reshape(m.ncell, nn), cfirst.reshape(m.ncell, nn)


@pytest.mark.parametrize("kind", [M.QUA8, M.TRI15, M.HEX8, M.TET4, M.HEX20])
def test_direct_assembly_replay_matches_the_oracle_bit_for_bit(kind):
    n = (4, 3, 1) if M.KIND_NDIM[kind] == 2 else (3, 2, 2)
    m = perturbed_mesh(kind, seed=1, n=n)
    prm = oracle.Params(2e5, 0.3, 1e3, 250.0)
    o = oracle.OracleElements(m, 1, prm, sym_tol=-1.0)
    o.initialize()
    o.update_secondary_values(plastic_ddu(m, seed=2))
    indptr, indices, ref = o.assemble_kk_csr()
    cslot, crank, cfirst = maps(m)
    nd, nn, ng = m.ndim, m.nnode, o.ngauss
    # block pattern from the scalar pattern: row A's block columns are its sorted neighbour nodes
    nb = [(indptr[nd * A + 1] - indptr[nd * A]) // nd for A in range(m.npoint)]
    bptr = np.concatenate([[0], np.cumsum(nb)])
    vals = np.full(len(ref), np.nan)  # untouched entries would stay NaN
    for c in range(m.ncell):  # ascending cell order, as the tickets enforce per row
        K = oracle.elem_jacobian(kind, ng, m.coords[m.cells[c]], 1, prm, o.sig[c * ng:(c + 1) * ng],
                                 o.ivs[c * ng:(c + 1) * ng], o.elastic[c * ng:(c + 1) * ng])
        for a in range(nn):
            A = m.cells[c, a]
            base, rs = nd * nd * bptr[A], nd * nb[A]
            for b in range(nn):
                first = (int(cfirst[c, a]) >> b) & 1
                assert first == ((int(cfirst[c, b]) >> a) & 1)  # symmetric in the pair
                for i in range(nd):
                    for j in range(nd):
                        pos = base + i * rs + nd * int(cslot[c, a, b]) + j
                        v = K[a * nd + i, b * nd + j]
                        vals[pos] = (0.0 + v) if first else vals[pos] + v
    assert not np.isnan(vals).any()
    assert np.array_equal(vals, ref)
    # ranks: per node, the cells in ascending order numbered 0, 1, ...; the last one flagged
    for A in range(m.npoint):
        cs, ls = np.nonzero(m.cells == A)
        r = crank[cs, ls]
        assert np.array_equal(r & (CRANK_LAST - 1), np.arange(len(cs)))
        assert np.array_equal((r & CRANK_LAST) != 0, np.arange(len(cs)) == len(cs) - 1)
