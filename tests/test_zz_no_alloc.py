"""The no-allocation entry point, pms_element_calc_noalloc, against the CPU oracle.

Callers that cannot call cudaMalloc (a framework that owns the whole device-memory budget, a
real-time loop that must not stall on an allocation, an FFI caller without a CUDA allocator) use
pms_element_calc_noalloc, which keeps its device data in one fixed file-scope array.  This test
calls it through the C ABI twice in a row (different cells and states, so the second call runs
over the first call's leftovers) and checks every cell's f and K against the oracle's element
vector and matrix (oracle.elem_f_int / oracle.elem_jacobian) on the same IP state, at the parity
tolerance of the other GPU tests.  The IP states come from the oracle's own stress update of a
plastic displacement increment.  The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from gpu_util import assert_close, perturbed_mesh, plastic_ddu
from pmsim_b200 import _lib
from pmsim_b200 import mesh as M

pytestmark = pytest.mark.gpu

E, NU, H, Z0 = 2e5, 0.3, 1e3, 250.0


def noalloc(kind, ngauss, X, sig, ivs, el, want_f=True, want_k=True):
    L = _lib.load()
    ncell, nn, nd = X.shape
    ne = nn * nd
    f = np.zeros((ncell, ne)) if want_f else None
    kk = np.zeros((ncell, ne, ne)) if want_k else None
    cap = ctypes.c_int64(-1)
    mat = _lib.material(_lib.VON_MISES, E, NU, H, Z0)
    rc = L.pms_element_calc_noalloc(kind, ngauss, 1.0, ctypes.byref(mat), ncell, _lib.ptr(np.ascontiguousarray(X)),
                                    _lib.ptr(np.ascontiguousarray(sig)), _lib.ptr(np.ascontiguousarray(ivs)),
                                    _lib.ptr(np.ascontiguousarray(el)), _lib.ptr(f), _lib.ptr(kk),
                                    ctypes.byref(cap), None)
    return rc, f, kk, cap.value


def oracle_case(kind, seed):
    """A perturbed mesh and the oracle's IP state after one plastic displacement increment."""
    m = perturbed_mesh(kind, seed=seed, n=(4, 3, 1) if M.KIND_NDIM[kind] == 2 else (3, 2, 2))
    o = oracle.OracleElements(m, oracle.MODEL_VON_MISES, oracle.Params(E, NU, H, Z0), sym_tol=-1.0)
    o.initialize()
    o.update_secondary_values(plastic_ddu(m, seed=seed))
    return m, o


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX20], ids=["qua8", "hex20"])
def test_noalloc_matches_oracle_two_calls(kind):
    params = oracle.Params(E, NU, H, Z0)
    for call, seed in enumerate((11, 12)):
        m, o = oracle_case(kind, seed)
        ng = o.ngauss
        cells = np.arange(m.ncell) if call == 0 else np.arange(m.ncell)[::-2]
        X = m.coords[m.cells[cells]]
        ips = (cells[:, None] * ng + np.arange(ng)[None, :]).ravel()
        sig, ivs, el = o.sig[ips], o.ivs[ips], o.elastic[ips]
        rc, f, kk, cap = noalloc(kind, 0, X, sig.T.copy(), ivs.T.copy(), el)
        assert rc == 0, rc
        assert cap >= len(cells)
        assert (1 - el.mean()) > 0  # plastic IPs present: the consistent tangent is exercised
        for i, c in enumerate(cells):
            s = slice(i * ng, (i + 1) * ng)
            kref = oracle.elem_jacobian(kind, ng, X[i], oracle.MODEL_VON_MISES, params, sig[s], ivs[s], el[s])
            fref = oracle.elem_f_int(kind, ng, X[i], sig[s])
            assert_close(kk[i], kref, what=f"call {call} K_e cell {c}")
            assert_close(f[i], fref, what=f"call {call} f_e cell {c}")


def test_noalloc_rejects_batches_beyond_the_scratch():
    kind = M.HEX20
    rc, _, _, cap = noalloc(kind, 0, np.zeros((0, 20, 3)), np.zeros((6, 0)), np.zeros((2, 0)),
                            np.zeros(0, np.uint8))
    assert rc == 0 and cap > 0
    n = cap + 1
    X = np.zeros((n, 20, 3))
    rc, _, _, cap2 = noalloc(kind, 0, X, np.zeros((6, n * 27)), np.zeros((2, n * 27)), np.ones(n * 27, np.uint8))
    assert rc == 8 and cap2 == cap  # PMS_ERR_TOO_LARGE, nothing launched
