"""The maps of the direct assembly (host only).  Replaying the device's order -- the cells in the
processing order of the maps, each block stored by the first of its cells and added to by the later
ones, at the slots of the maps -- with the oracle's element matrices: every first contribution lands
on an untouched entry and every later one on a written entry, and the result equals the oracle's
CSR values (the reference's COO duplicates summed in ascending cell order) to rounding.  Also checks
the ranks that order the row slabs, and that the processing order is a permutation in colour
classes that keeps disjoint meshes in their own cell ranges (the batched solver's problems)."""
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
    order = np.zeros(m.ncell, np.int32)
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    assert L.pms_mesh_assembly_maps(ctypes.byref(cm), _lib.ptr(cslot), _lib.ptr(crank), _lib.ptr(cfirst),
                                    _lib.ptr(order)) == 0
    return cslot.reshape(m.ncell, nn, nn), crank.reshape(m.ncell, nn), cfirst.reshape(m.ncell, nn), order


@pytest.mark.parametrize("kind", [M.QUA8, M.TRI15, M.HEX8, M.TET4, M.HEX20])
def test_direct_assembly_replay_matches_the_oracle_bit_for_bit(kind):
    n = (4, 3, 1) if M.KIND_NDIM[kind] == 2 else (3, 2, 2)
    m = perturbed_mesh(kind, seed=1, n=n)
    prm = oracle.Params(2e5, 0.3, 1e3, 250.0)
    o = oracle.OracleElements(m, 1, prm, sym_tol=-1.0)
    o.initialize()
    o.update_secondary_values(plastic_ddu(m, seed=2))
    indptr, indices, ref = o.assemble_kk_csr()
    cslot, crank, cfirst, order = maps(m)
    assert np.array_equal(np.sort(order), np.arange(m.ncell))
    nd, nn, ng = m.ndim, m.nnode, o.ngauss
    # block pattern from the scalar pattern: row A's block columns are its sorted neighbour nodes
    nb = [(indptr[nd * A + 1] - indptr[nd * A]) // nd for A in range(m.npoint)]
    bptr = np.concatenate([[0], np.cumsum(nb)])
    vals = np.full(len(ref), np.nan)  # untouched entries stay NaN
    for c in order:  # the processing order, as the tickets enforce per row
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
                        assert np.isnan(vals[pos]) == bool(first)
                        vals[pos] = (0.0 + v) if first else vals[pos] + v
    assert not np.isnan(vals).any()
    assert np.abs(vals - ref).max() <= 1e-14 * np.abs(ref).max()
    # ranks: per node, its cells in the processing order numbered 0, 1, ...; the last one flagged
    opos = np.empty(m.ncell, np.int64)
    opos[order] = np.arange(m.ncell)
    for A in range(m.npoint):
        cs, ls = np.nonzero(m.cells == A)
        srt = np.argsort(opos[cs])
        r = crank[cs[srt], ls[srt]]
        assert np.array_equal(r & (CRANK_LAST - 1), np.arange(len(cs)))
        assert np.array_equal((r & CRANK_LAST) != 0, np.arange(len(cs)) == len(cs) - 1)
    # colour classes: cells taken one after another share no node, except where a class ends
    share = sum(bool(np.intersect1d(m.cells[order[k]], m.cells[order[k + 1]]).size) for k in range(m.ncell - 1))
    assert share <= 27


def test_processing_order_keeps_disjoint_meshes_in_their_ranges():
    a = M.structured_2d(M.QUA8, 5, 4)
    b = M.structured_2d(M.QUA8, 3, 6, x0=10.0)
    m = M.Mesh(2, np.vstack([a.coords, b.coords]), np.vstack([a.cells, b.cells + a.npoint]), M.QUA8)
    _, _, _, order = maps(m)
    assert np.array_equal(np.sort(order[:a.ncell]), np.arange(a.ncell))
    assert np.array_equal(np.sort(order[a.ncell:]), np.arange(a.ncell, m.ncell))
    assert not np.array_equal(order, np.arange(m.ncell))  # the colours do reorder each mesh
