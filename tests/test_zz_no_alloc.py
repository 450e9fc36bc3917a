"""The no-allocation entry point, pms_element_calc_noalloc, against the handle-based path.

Callers that cannot call cudaMalloc (a framework that owns the whole device-memory budget, a
real-time loop that must not stall on an allocation, an FFI caller without a CUDA allocator) use
pms_element_calc_noalloc, which keeps its device data in one fixed file-scope array.  This test
calls it through the C ABI twice in a row (different cells and states, so the second call runs
over the first call's leftovers) and checks f and K against pms_element_calc_f_int /
pms_element_calc_jacobian of an Elements handle, at the parity tolerance of the other GPU tests.
The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

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


def handle_case(kind, seed):
    from pmsim_b200.elements import Elements, Material
    m = perturbed_mesh(kind, seed=seed, n=(4, 3, 1) if M.KIND_NDIM[kind] == 2 else (3, 2, 2))
    g = Elements(m, Material.von_mises(E, NU, H, Z0))
    g.initialize_internal_values()
    g.update_secondary_values(plastic_ddu(m, seed=seed))
    return m, g


@pytest.mark.parametrize("kind", [M.QUA8, M.HEX20], ids=["qua8", "hex20"])
def test_noalloc_matches_handle_path_two_calls(kind):
    for call, seed in enumerate((11, 12)):
        m, g = handle_case(kind, seed)
        sig, ivs, el = g.get_state()
        ng, nc = g.ngauss, g.ncomp
        cells = np.arange(m.ncell) if call == 0 else np.arange(m.ncell)[::-2]
        X = m.coords[m.cells[cells]]
        ips = (cells[:, None] * ng + np.arange(ng)[None, :]).ravel()
        rc, f, kk, cap = noalloc(kind, 0, X, sig[ips].T.copy(), ivs[ips].T.copy(), el[ips])
        assert rc == 0, rc
        assert cap >= len(cells)
        assert (1 - el[ips].mean()) > 0  # plastic IPs present: the consistent tangent is exercised
        for i, c in enumerate(cells):
            assert_close(kk[i], g.calc_jacobian(int(c)), what=f"call {call} K_e cell {c}")
            assert_close(f[i], g.calc_f_int(int(c)), what=f"call {call} f_e cell {c}")


def test_noalloc_rejects_batches_beyond_the_scratch():
    kind = M.HEX20
    rc, _, _, cap = noalloc(kind, 0, np.zeros((0, 20, 3)), np.zeros((6, 0)), np.zeros((2, 0)),
                            np.zeros(0, np.uint8))
    assert rc == 0 and cap > 0
    n = cap + 1
    X = np.zeros((n, 20, 3))
    rc, _, _, cap2 = noalloc(kind, 0, X, np.zeros((6, n * 27)), np.zeros((2, n * 27)), np.ones(n * 27, np.uint8))
    assert rc == 8 and cap2 == cap  # PMS_ERR_TOO_LARGE, nothing launched
