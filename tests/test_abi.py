"""C-ABI checks that need no GPU: the library loads, exports every symbol include/pms.h declares,
and the host-only CSR pattern equals the oracle's COO->CSR pattern."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from pmsim_b200 import _lib
from pmsim_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(pms_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) == names


def test_version_string():
    assert b"sm_100a" in _lib.load().pms_version()


@pytest.mark.parametrize("kind", [M.TRI3, M.TRI6, M.QUA4, M.QUA8, M.QUA9, M.TET4, M.HEX8, M.HEX20])
def test_host_csr_pattern_matches_oracle(kind):
    if M.KIND_NDIM[kind] == 2:
        m = M.structured_2d(kind, 3, 2, 3.0, 2.0)
    else:
        m = M.structured_3d(kind, 2, 2, 1)
    L = _lib.load()
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    nnz = ctypes.c_int64()
    indptr = np.zeros(m.ndof + 1, np.int64)
    assert L.pms_mesh_csr_pattern(ctypes.byref(cm), _lib.ptr(indptr), None, ctypes.byref(nnz)) == 0
    indices = np.zeros(nnz.value, np.int32)
    assert L.pms_mesh_csr_pattern(ctypes.byref(cm), _lib.ptr(indptr), _lib.ptr(indices), ctypes.byref(nnz)) == 0
    o = oracle.OracleElements(m, 0, oracle.Params(1.0, 0.3))
    o.initialize()
    ip, ix, _ = o.assemble_kk_csr()
    assert np.array_equal(ip, indptr) and np.array_equal(ix, indices)


@pytest.mark.parametrize("kind", [M.TRI3, M.QUA8, M.TET4, M.HEX8, M.HEX20])
def test_host_triangle_patterns(kind):
    """Sym::YesLower / YesUpper storage (src/base/assembly.rs:92-122): the full pattern's entries with
    column <= row (lower) or >= row (upper), in order; a symmetric pattern keeps its diagonal and
    half of the rest."""
    if M.KIND_NDIM[kind] == 2:
        m = M.structured_2d(kind, 4, 3, 4.0, 3.0)
    else:
        m = M.structured_3d(kind, 2, 2, 2)
    L = _lib.load()
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    o = oracle.OracleElements(m, 0, oracle.Params(1.0, 0.3))
    o.initialize()
    ip, ix, _ = o.assemble_kk_csr()
    rows = np.repeat(np.arange(m.ndof), np.diff(ip))
    for sym, keep in ((_lib.PMS_SYM_LOWER, ix <= rows), (_lib.PMS_SYM_UPPER, ix >= rows)):
        nnz = ctypes.c_int64()
        assert L.pms_mesh_csr_pattern_sym(ctypes.byref(cm), sym, None, None, ctypes.byref(nnz)) == 0
        assert nnz.value == int(keep.sum()) and 2 * nnz.value - m.ndof == len(ix)
        indptr = np.zeros(m.ndof + 1, np.int64)
        indices = np.zeros(nnz.value, np.int32)
        assert L.pms_mesh_csr_pattern_sym(ctypes.byref(cm), sym, _lib.ptr(indptr), _lib.ptr(indices), None) == 0
        assert np.array_equal(indices, ix[keep])
        assert np.array_equal(np.diff(indptr), np.bincount(rows[keep], minlength=m.ndof))
    assert L.pms_mesh_csr_pattern_sym(ctypes.byref(cm), 3, None, None, None) == _lib.PMS_ERR_INVALID


def test_hex20_block_sizes_of_the_large_problem():
    """64x64x32 Hex20: 549,185 points, 1,647,555 DOF, nnz 279,514,377 (host pattern, no GPU)."""
    m = M.structured_3d(M.HEX20, 64, 64, 32, 64.0, 64.0, 32.0)
    assert (m.npoint, m.ncell, m.ndof) == (549185, 131072, 1647555)
    L = _lib.load()
    cm = _lib.Mesh_(m.ndim, m.kind, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    nnz = ctypes.c_int64()
    assert L.pms_mesh_csr_pattern(ctypes.byref(cm), None, None, ctypes.byref(nnz)) == 0
    assert nnz.value == 279514377
    assert L.pms_mesh_csr_pattern_sym(ctypes.byref(cm), _lib.PMS_SYM_LOWER, None, None, ctypes.byref(nnz)) == 0
    assert nnz.value == (279514377 + 1647555) // 2  # 140,580,966 values of MUMPS's lower triangle


def test_invalid_arguments_are_rejected_without_gpu():
    L = _lib.load()
    bad = _lib.Mesh_(2, 99, 4, 1, None, None, None)
    assert L.pms_mesh_csr_pattern(ctypes.byref(bad), None, None, None) == 1
    m = M.structured_2d(M.QUA4, 1, 1)
    cells = m.cells.copy()
    cells[0, 0] = 100  # point out of range
    cm = _lib.Mesh_(2, M.QUA4, m.npoint, 1, _lib.ptr(m.coords), _lib.ptr(cells), None)
    assert L.pms_mesh_csr_pattern(ctypes.byref(cm), None, None, None) == 1


def test_unsupported_idealizations_are_rejected_without_gpu():
    """Plane stress with von Mises is refused as the reference refuses it ("von Mises model does not
    work in plane-stress", src/material/von_mises.rs:60-62), and so are 3D axisymmetric or plane-stress
    configurations; these checks come before any device work."""
    L = _lib.load()
    m = M.structured_2d(M.QUA4, 1, 1)
    cm = _lib.Mesh_(2, M.QUA4, m.npoint, m.ncell, _lib.ptr(m.coords), _lib.ptr(m.cells), None)
    vm = _lib.material(_lib.VON_MISES, 1e4, 0.3, 0.0, 9.0)
    h = ctypes.c_void_p()
    assert L.pms_elements_create(ctypes.byref(cm), ctypes.byref(vm), 1, ctypes.byref(_lib.Config_(0, 1, 0, 1.0)),
                                 ctypes.byref(h)) == 7
    m3 = M.structured_3d(M.HEX8, 1, 1, 1)
    cm3 = _lib.Mesh_(3, M.HEX8, m3.npoint, m3.ncell, _lib.ptr(m3.coords), _lib.ptr(m3.cells), None)
    le = _lib.material(_lib.LINEAR_ELASTIC, 1e4, 0.3, 0.0, 1.0)
    for cfg in (_lib.Config_(0, 1, 0, 1.0), _lib.Config_(0, 0, 1, 1.0)):
        assert L.pms_elements_create(ctypes.byref(cm3), ctypes.byref(le), 1, ctypes.byref(cfg), ctypes.byref(h)) == 7


def test_general_elastoplastic_rejects_other_models_without_gpu():
    """Elastoplastic::new accepts only the von Mises plasticity model (elastoplastic.rs:129-135):
    the batched entry refuses a linear-elastic material and bad sizes before touching the GPU."""
    L = _lib.load()
    s = _lib.EpSettings_(1e-10, 1e-10, 1.0, 1000, 0)
    lin = _lib.material(_lib.LINEAR_ELASTIC, 1500.0, 0.25, 0.0, 1.0)
    vm = _lib.material(_lib.VON_MISES, 1500.0, 0.25, 800.0, 9.0)
    assert L.pms_ep_update_stress_batch(ctypes.byref(lin), 2, 1, None, None, None, None, ctypes.byref(s),
                                        None, None, None, None) == 1
    assert L.pms_ep_update_stress_batch(ctypes.byref(vm), 4, 1, None, None, None, None, ctypes.byref(s),
                                        None, None, None, None) == 1
    assert L.pms_ep_update_stress_batch(ctypes.byref(vm), 2, 0, None, None, None, None, ctypes.byref(s),
                                        None, None, None, None) == 0
    bad = _lib.EpSettings_(0.0, 1e-10, 1.0, 1000, 0)
    assert L.pms_ep_update_stress_batch(ctypes.byref(vm), 2, 1, None, None, None, None, ctypes.byref(bad),
                                        None, None, None, None) == 1


def test_shape_tables_match_the_oracle_for_every_kind():
    """pms_shape_table (the tables pms_elements_create uploads) against the oracle's Gauss rules and
    shape functions, every kind and its default rule plus the alternative rules (host only)."""
    import ctypes

    import numpy as np

    import oracle
    from pmsim_b200 import mesh as M
    L = _lib.load()
    rules = {k: [0] for k in range(len(M.KIND_NAMES))}
    rules[M.QUA8] += [4, 9]
    rules[M.TRI6] += [6, 7, 12]
    rules[M.TRI15] += [6, 7]
    rules[M.HEX8] += [27]
    for kind, ngs in rules.items():
        nn, nd = M.KIND_NNODE[kind], M.KIND_NDIM[kind]
        for ngauss in ngs:
            ng = ctypes.c_int32(0)
            assert L.pms_shape_table(kind, ngauss, None, ctypes.byref(ng)) == 0, (kind, ngauss)
            n = ng.value
            tab = np.zeros(n * nn * nd + n + n * nn)
            assert L.pms_shape_table(kind, ngauss, _lib.ptr(tab), None) == 0
            ksi, w = oracle.gauss(kind, ngauss)
            assert len(w) == n, (kind, ngauss)
            np.testing.assert_allclose(tab[n * nn * nd:n * nn * nd + n], w, rtol=0, atol=1e-15)
            for p in range(n):
                N, dN = oracle.shape(kind, ksi[p][:nd])
                np.testing.assert_allclose(tab[p * nn * nd:(p + 1) * nn * nd], dN[:nn * nd], rtol=0, atol=1e-13)
                off = n * nn * nd + n + p * nn
                np.testing.assert_allclose(tab[off:off + nn], N[:nn], rtol=0, atol=1e-14)
    assert L.pms_shape_table(99, 0, None, None) != 0


def test_dpcg_create_refuses_bad_input_before_any_device_call():
    """pms_dpcg_create checks its host arrays before touching the device (host only)."""
    import ctypes

    import numpy as np
    L = _lib.load()
    ip = np.array([0, 1, 2], dtype=np.int64)
    ix = np.array([0, 5], dtype=np.int32)  # column 5 is outside the 4 local DOFs
    fx = np.zeros(4, dtype=np.uint8)
    h = ctypes.c_void_p()
    assert L.pms_dpcg_create(4, 2, 4, _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(fx), 0, None, 0, None,
                             ctypes.byref(h)) == _lib.PMS_ERR_INVALID
    assert b"ndim" in L.pms_dpcg_last_error(None)
    assert L.pms_dpcg_create(2, 2, 4, _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(fx), 0, None, 0, None,
                             ctypes.byref(h)) == _lib.PMS_ERR_INVALID
    assert b"column" in L.pms_dpcg_last_error(None)
    ix[1] = 1
    bad_recv = np.array([0], dtype=np.int64)  # an owned DOF is not a ghost
    assert L.pms_dpcg_create(2, 2, 4, _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(fx), 0, None, 1, _lib.ptr(bad_recv),
                             ctypes.byref(h)) == _lib.PMS_ERR_INVALID
    assert b"ghost" in L.pms_dpcg_last_error(None)
    assert h.value is None
