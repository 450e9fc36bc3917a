"""The host plan for assembling element blocks straight into the CSR values
(pmsim_b200/assembly_plan.py): a valid colouring, row-budgeted chunks, and block slots that put
every element block where the assembled matrix has it -- checked by applying the plan on the host
to the oracle's element matrices and comparing with the oracle's assembled K."""
import numpy as np
import pytest

import oracle
from pmsim_b200 import assembly_plan as P
from pmsim_b200.mesh import HEX8, QUA8, structured_2d, structured_3d

E, NU, H, Z0 = 1e4, 0.3, 500.0, 9.0


def _mesh(kind):
    m = structured_3d(HEX8, 3, 2, 2, 1.5, 1.0, 1.0) if kind == HEX8 else structured_2d(QUA8, 6, 4, 3.0, 2.0)
    rng = np.random.default_rng(kind + 5)
    inner = np.all((m.coords > 1e-9) & (m.coords < m.coords.max(axis=0) - 1e-9), axis=1)
    m.coords[inner] += rng.uniform(-0.05, 0.05, (inner.sum(), m.ndim))
    return m


@pytest.mark.parametrize("kind,ncolor", [(QUA8, 4), (HEX8, 8)])
def test_plan_reproduces_the_assembled_matrix(kind, ncolor):
    m = _mesh(kind)
    nd = m.ndim
    colors, nc = P.color_cells(m)
    assert nc == ncolor
    for k in range(nc):  # cells of one colour share no node
        nodes = m.cells[colors == k].ravel()
        assert len(nodes) == len(np.unique(nodes))
    order, chunk_ptr, color_ptr = P.chunk_cells(m, colors, max_rows=40)
    assert np.array_equal(np.sort(order), np.arange(m.ncell))
    for k in range(len(chunk_ptr) - 1):
        chunk = order[chunk_ptr[k]:chunk_ptr[k + 1]]
        assert len(np.unique(m.cells[chunk])) <= 40 or len(chunk) == 1
        assert np.all(np.diff(colors[chunk]) >= 0)
        assert color_ptr[k][0] == chunk_ptr[k] and color_ptr[k][-1] == chunk_ptr[k + 1]
    # element matrices on a plastic state, and the assembled K, from the oracle
    prm = oracle.Params(E, NU, H, Z0)
    el = oracle.OracleElements(m, oracle.MODEL_VON_MISES, prm, sym_tol=-1.0)
    el.initialize()
    rng = np.random.default_rng(kind)
    u = np.zeros((m.npoint, nd))
    u[:, -1] = -0.003 * m.coords[:, -1] * (1.0 + np.sin(2.0 * m.coords[:, 0]))
    el.update_secondary_values((u + rng.normal(0.0, 1e-4, u.shape)).reshape(-1))
    assert el.elastic.min() == 0
    ip, ix, vals = el.assemble_kk_csr()
    ng = el.ngauss
    ke = np.array([oracle.elem_jacobian(m.kind, ng, m.coords[m.cells[c]], oracle.MODEL_VON_MISES, prm,
                                        el.sig[c * ng:(c + 1) * ng], el.ivs[c * ng:(c + 1) * ng],
                                        el.elastic[c * ng:(c + 1) * ng]) for c in range(m.ncell)])
    bptr, bcol = P.block_pattern(ip, ix, nd)
    slots = P.block_slots(m, bptr, bcol)
    got = P.emulate(m, ke, bptr, slots, order)
    scale = np.abs(vals).max()
    assert np.max(np.abs(got - vals)) <= 1e-13 * scale
    # another valid order gives the same matrix up to rounding, the same order the same bits
    again = P.emulate(m, ke, bptr, slots, order)
    assert np.array_equal(got, again)
    other = P.emulate(m, ke, bptr, slots, np.arange(m.ncell)[::-1])
    assert np.max(np.abs(other - got)) <= 1e-13 * scale


def test_block_slots_refuse_a_pattern_without_the_cell_block():
    """A pattern that lacks one of a cell's node blocks is refused, not mapped to a neighbouring slot."""
    m = _mesh(QUA8)
    ip, ix, _ = oracle.coo_to_csr(m.ndof, *[np.asarray(a) for a in _coo(m)])
    bptr, bcol = P.block_pattern(ip, ix, m.ndim)
    P.block_slots(m, bptr, bcol)  # the full pattern maps every block
    A, B = int(m.cells[0, 0]), int(m.cells[0, 2])
    row = bcol[bptr[A]:bptr[A + 1]]
    keep = np.ones(len(bcol), bool)
    keep[bptr[A] + int(np.flatnonzero(row == B)[0])] = False
    bcol2 = bcol[keep]
    bptr2 = bptr.copy()
    bptr2[A + 1:] -= 1
    with pytest.raises(ValueError):
        P.block_slots(m, bptr2, bcol2)


def _coo(m):
    """Unit entries at every (cell node, cell node) DOF pair: the pattern of K."""
    nd, nn = m.ndim, m.nnode
    dofs = (m.cells[:, :, None] * nd + np.arange(nd)).reshape(m.ncell, nn * nd)
    rows = np.repeat(dofs, nn * nd, axis=1).ravel().astype(np.int64)
    cols = np.tile(dofs, (1, nn * nd)).ravel().astype(np.int64)
    return rows, cols, np.ones(rows.size)
