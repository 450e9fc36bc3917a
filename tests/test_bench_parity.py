"""The bench's parity check of the GPU step (bench.parity_sample), exercised on the CPU: the oracle
over the whole mesh stands in for the GPU and must pass against the oracle over the first cells;
mistakes planted in that stand-in (a stress, an R entry, a CSR value, a flag) must fail it."""
import numpy as np

import bench
import oracle
from gpu_util import plastic_ddu
from pmsim_b200 import mesh as M


def _full_and_sample():
    m = M.structured_3d(M.HEX20, 4, 4, 3, 4.0, 4.0, 3.0)
    ddu = plastic_ddu(m, seed=3, strain=6e-4)
    full = oracle.OracleElements(m, oracle.MODEL_VON_MISES, oracle.Params(bench.E, bench.NU, bench.HH, bench.Z0),
                                 sym_tol=-1.0)
    full.initialize()
    full.update_secondary_values(ddu)
    ff = full.assemble_f_int()
    indptr, indices, vals = full.assemble_kk_csr()
    ncs = 24
    _, _, ref = bench.cpu_sample(m, ddu, ncs, 1)
    return m, ncs, (full.sig.copy(), full.ivs.copy(), full.elastic.copy()), ff, vals, indptr, indices, ref


def test_parity_sample_passes_on_the_same_arithmetic_and_fails_on_planted_mistakes():
    m, ncs, state, ff, vals, indptr, indices, ref = _full_and_sample()
    out = bench.parity_sample(m, ncs, state, ff, vals, indptr, indices, ref)
    assert out["ok"], out
    assert out["rows_compared"] > 0 and out["csr_values_compared"] > 0
    assert 0 < 1 - state[2][: ncs * 27].mean() < 1
    oel = ref[0]
    inside_row = int(np.flatnonzero(np.abs(ref[1]) > 0)[0])
    # which CSR values lie in compared rows: perturb one of them
    n_all = np.bincount(m.cells.ravel(), minlength=m.npoint)
    n_in = np.bincount(m.cells[:ncs].ravel(), minlength=m.npoint)
    node = int(np.flatnonzero((n_all == n_in) & (n_in > 0))[0])
    row = 3 * node
    for what in ("sigma", "f_int", "csr", "flag"):
        sig, ivs, el = (a.copy() for a in state)
        f2, v2 = ff.copy(), vals.copy()
        if what == "sigma":
            sig[5, 1] *= 1 + 1e-9
        elif what == "f_int":
            f2[row] += 1e-9 * np.abs(ff).max()
        elif what == "csr":
            v2[indptr[row]] *= 1 + 1e-9
        else:
            el[7] ^= 1
        out = bench.parity_sample(m, ncs, (sig, ivs, el), f2, v2, indptr, indices, ref)
        assert not out["ok"], what
    assert inside_row >= 0 and oel.ngauss == 27
