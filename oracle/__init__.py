"""CPU parity oracle for the pmsim solid hot path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this package, and only as the checker (or the timed CPU restatement).  The product
(``pmsim_b200``) never imports it.

``libpms_oracle.so`` (built from ``pms_oracle.cpp`` by ``make -C oracle``) restates the
reference's element/material arithmetic; ``driver.py`` restates its Newton/time loop.
Parity is pinned against the reference's own golden data: the inline von Mises KATs
(``src/material/von_mises.rs:324-480``) and the SPO/HYPLAS runs (``data/spo/*.json``),
committed as fixtures under ``tests/golden/``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int64_p = ctypes.POINTER(ctypes.c_int64)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)
c_int_p = ctypes.POINTER(ctypes.c_int)

MODEL_LINEAR_ELASTIC = 0
MODEL_VON_MISES = 1
MODEL_LINEAR_ELASTIC_PLANE_STRESS = 2  # 2D only


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libpms_oracle.so")
        src = os.path.join(_HERE, "pms_oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        L.orc_gauss.argtypes = [ctypes.c_int, ctypes.c_int, c_double_p, c_double_p]
        L.orc_shape.argtypes = [ctypes.c_int, c_double_p, c_double_p, c_double_p]
        L.orc_model_update_stress.argtypes = [ctypes.c_int, c_double_p, ctypes.c_int, c_double_p, c_double_p,
                                              c_uint8_p, c_double_p]
        L.orc_model_stiffness.argtypes = [ctypes.c_int, c_double_p, ctypes.c_int, c_double_p, c_double_p,
                                          ctypes.c_uint8, c_double_p]
        L.orc_model_update_and_stiffness_batch.argtypes = [ctypes.c_int, c_double_p, ctypes.c_int, ctypes.c_int64,
                                                           c_double_p, c_double_p, c_uint8_p, c_double_p,
                                                           c_double_p, ctypes.c_int]
        L.orc_model_batch_hh.argtypes = [ctypes.c_int, c_double_p, ctypes.c_int, ctypes.c_int64, c_double_p,
                                          c_double_p, c_double_p, c_uint8_p, c_double_p, c_double_p, ctypes.c_int]
        L.orc_elem_f_int.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, c_double_p, c_double_p,
                                     c_double_p]
        L.orc_elem_jacobian.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, c_double_p, ctypes.c_int,
                                        c_double_p, c_double_p, c_double_p, c_uint8_p, c_double_p]
        L.orc_assemble_f_int.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int64, c_double_p,
                                         ctypes.c_int64, c_int64_p, c_double_p, c_double_p]
        L.orc_assemble_kk_coo.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, c_double_p, ctypes.c_int64,
                                          c_int64_p, ctypes.c_int, c_double_p, c_double_p, c_double_p, c_uint8_p,
                                          ctypes.c_double, c_int64_p, c_int64_p, c_double_p, ctypes.c_int,
                                          c_int64_p]
        L.orc_coo_to_csr.argtypes = [ctypes.c_int64, ctypes.c_int64, c_int64_p, c_int64_p, c_double_p, c_int64_p,
                                     c_int64_p, c_double_p]
        L.orc_coo_to_csr.restype = ctypes.c_int64
        L.orc_ep_update_batch.argtypes = [c_double_p, ctypes.c_int, ctypes.c_int64, c_double_p, c_double_p,
                                          c_uint8_p, c_double_p, c_double_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                          c_int64_p]
        L.orc_update_secondary.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, c_double_p, ctypes.c_int64,
                                           c_int64_p, ctypes.c_int, c_double_p, c_double_p, c_double_p, c_double_p,
                                           c_uint8_p, ctypes.c_int, c_int64_p, c_int_p]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


def _dp(a):
    return _p(a, c_double_p)


def gauss(kind, ngauss=0):
    ksi = np.zeros((27, 3))
    w = np.zeros(27)
    n = lib().orc_gauss(kind, ngauss, _dp(ksi), _dp(w))
    if n <= 0:
        raise ValueError("requested number of integration points is not available")
    return ksi[:n].copy(), w[:n].copy()


def shape(kind, ksi):
    ksi = np.ascontiguousarray(np.pad(np.asarray(ksi, float), (0, 3 - len(ksi))))
    N = np.zeros(20)
    dN = np.zeros(60)
    lib().orc_shape(kind, _dp(ksi), _dp(N), _dp(dN))
    return N, dN


class Params:
    """Von Mises / linear elastic parameters [young, poisson, hh, z_ini]."""

    def __init__(self, young, poisson, hh=0.0, z_ini=1.0):
        self.arr = np.array([young, poisson, hh, z_ini], dtype=np.float64)


def model_update_stress(model, params, ndim, sig, ivs, elastic, deps):
    """In-place update of one IP state (sig: nc, ivs: [z, lambda], elastic: uint8[1])."""
    st = lib().orc_model_update_stress(model, _dp(params.arr), ndim, _dp(sig), _dp(ivs), _p(elastic, c_uint8_p),
                                       _dp(np.ascontiguousarray(deps, dtype=np.float64)))
    return st


def model_stiffness(model, params, ndim, sig, ivs, elastic):
    nc = 2 * ndim
    dd = np.zeros((nc, nc))
    st = lib().orc_model_stiffness(model, _dp(params.arr), ndim, _dp(sig), _dp(ivs), int(elastic), _dp(dd))
    if st:
        raise RuntimeError(f"stiffness error {st}")
    return dd


def model_batch(model, params, ndim, sig, ivs, elastic, deps, with_tangent=True, nthreads=1):
    """Batched update (+ tangent) over n IPs; AoS arrays updated in place. Returns dd or None."""
    n = sig.shape[0]
    nc = 2 * ndim
    dd = np.zeros((n, nc, nc)) if with_tangent else None
    st = lib().orc_model_update_and_stiffness_batch(model, _dp(params.arr), ndim, n, _dp(sig), _dp(ivs),
                                                    _p(elastic, c_uint8_p), _dp(deps), _dp(dd), nthreads)
    if st:
        raise RuntimeError(f"material batch error {st}")
    return dd


def model_batch_hh(model, params, ndim, hh, sig, ivs, elastic, deps, nthreads=0):
    """model_batch with a hardening modulus per IP (hh[n]); returns the tangents (n, nc, nc)."""
    n = sig.shape[0]
    nc = 2 * ndim
    dd = np.zeros((n, nc, nc))
    st = lib().orc_model_batch_hh(model, _dp(params.arr), ndim, n, _dp(np.ascontiguousarray(hh, dtype=np.float64)),
                                  _dp(sig), _dp(ivs), _p(elastic, c_uint8_p), _dp(deps), _dp(dd), nthreads)
    if st:
        raise RuntimeError(f"material batch error {st}")
    return dd


EP_CASES = ("AE", "AXB", "BE", "BXP", "BP")


def ep_update(params, ndim, sig, z, elastic, deps, tol_rel=1e-10, tol_abs=1e-10, h_ini=1.0, max_steps=1000):
    """General elastoplastic update (Elastoplastic::update_stress with the von Mises model) of n
    IPs in place: sig (n, nc), z (n), elastic (n, uint8), deps (n, nc).  Returns (code, cases,
    steps, first failing IP or -1)."""
    n = sig.shape[0]
    cases = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int32)
    bad = np.array([-1], dtype=np.int64)
    st = lib().orc_ep_update_batch(_dp(params.arr), ndim, n, _dp(sig), _dp(z), _p(elastic, c_uint8_p),
                                   _dp(np.ascontiguousarray(deps, dtype=np.float64)),
                                   _dp(np.array([tol_rel, tol_abs, h_ini], dtype=np.float64)), max_steps,
                                   cases.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   steps.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   bad.ctypes.data_as(c_int64_p))
    return st, cases, steps, int(bad[0])


def elem_f_int(kind, ngauss, X, sig, thickness=1.0):
    X = np.ascontiguousarray(X, dtype=np.float64)
    f = np.zeros(X.size)
    st = lib().orc_elem_f_int(kind, ngauss, thickness, _dp(X), _dp(np.ascontiguousarray(sig)), _dp(f))
    if st:
        raise RuntimeError(f"f_int error {st}")
    return f


def elem_jacobian(kind, ngauss, X, model, params, sig, ivs, elastic, thickness=1.0):
    X = np.ascontiguousarray(X, dtype=np.float64)
    ne = X.size
    K = np.zeros((ne, ne))
    st = lib().orc_elem_jacobian(kind, ngauss, thickness, _dp(X), model, _dp(params.arr),
                                 _dp(np.ascontiguousarray(sig)), _dp(np.ascontiguousarray(ivs)),
                                 _p(np.ascontiguousarray(elastic, dtype=np.uint8), c_uint8_p), _dp(K))
    if st:
        raise RuntimeError(f"jacobian error {st}")
    return K


class OracleError(RuntimeError):
    """An element-loop error with the failing cell (and IP, for the stress update), as the
    reference's loops report the first one (src/fem/elements.rs:156-181)."""

    def __init__(self, msg, code, cell, ip=-1):
        super().__init__(msg)
        self.code, self.cell, self.ip = code, cell, ip


class OracleElements:
    """Mirror of ``Elements`` (src/fem/elements.rs) over a homogeneous mesh, AoS IP state."""

    def __init__(self, mesh, model, params, ngauss=0, thickness=1.0, sym_tol=1e-10, nthreads=1, axisymmetric=False):
        self.mesh = mesh
        self.kind = mesh.kind
        self.model = model
        self.params = params
        self.ngauss = ngauss if ngauss > 0 else lib().orc_default_ngauss(mesh.kind)
        self.thickness = -1.0 if axisymmetric else thickness  # < 0: axisymmetric (weight = radius)
        self.sym_tol = sym_tol
        self.nthreads = nthreads
        self.nc = 2 * mesh.ndim
        nip = mesh.ncell * self.ngauss
        self.sig = np.zeros((nip, self.nc))
        self.ivs = np.zeros((nip, 2))
        self.elastic = np.ones(nip, dtype=np.uint8)
        self.backup = None

    # ElementTrait::initialize_internal_values (von_mises.rs:107-116)
    def initialize(self):
        self.sig[:] = 0.0
        self.ivs[:, 0] = self.params.arr[3] if self.model == MODEL_VON_MISES else 0.0
        self.ivs[:, 1] = 0.0
        self.elastic[:] = 1

    def reset_algorithmic_variables(self):
        if self.model == MODEL_VON_MISES:
            self.ivs[:, 1] = 0.0

    def backup_secondary_values(self):
        self.backup = (self.sig.copy(), self.ivs.copy(), self.elastic.copy())

    def restore_secondary_values(self):
        s, i, e = self.backup
        self.sig[:] = s
        self.ivs[:] = i
        self.elastic[:] = e

    def assemble_f_int(self):
        m = self.mesh
        ff = np.zeros(m.ndof)
        st = lib().orc_assemble_f_int(self.kind, self.ngauss, self.thickness, m.npoint, _dp(m.coords), m.ncell,
                                      _p(m.cells, c_int64_p), _dp(self.sig), _dp(ff))
        if st:
            raise OracleError(f"assemble_f_int error {st}", st, -1)
        return ff

    def assemble_kk_coo(self):
        m = self.mesh
        ne = m.nnode * m.ndim
        ntrip = m.ncell * ne * ne
        rows = np.empty(ntrip, np.int64)
        cols = np.empty(ntrip, np.int64)
        vals = np.empty(ntrip)
        bad = np.zeros(1, np.int64)
        st = lib().orc_assemble_kk_coo(self.kind, self.ngauss, self.thickness, _dp(m.coords), m.ncell,
                                       _p(m.cells, c_int64_p), self.model, _dp(self.params.arr), _dp(self.sig),
                                       _dp(self.ivs), _p(self.elastic, c_uint8_p), self.sym_tol,
                                       _p(rows, c_int64_p), _p(cols, c_int64_p), _dp(vals), self.nthreads,
                                       _p(bad, c_int64_p))
        if st == 5:
            raise OracleError("local matrix is not symmetric", st, int(bad[0]))
        if st == 3:
            raise OracleError("von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)",
                              st, int(bad[0]))
        if st:
            raise OracleError(f"assemble_kk error {st} at cell {bad[0]}", st, int(bad[0]))
        return rows, cols, vals

    def assemble_kk_csr(self):
        rows, cols, vals = self.assemble_kk_coo()
        return coo_to_csr(self.mesh.ndof, rows, cols, vals)

    def update_secondary_values(self, ddu):
        m = self.mesh
        ddu = np.ascontiguousarray(ddu[: m.ndof], dtype=np.float64)
        bc = np.zeros(1, np.int64)
        bi = np.zeros(1, np.int32)
        st = lib().orc_update_secondary(self.kind, self.ngauss, self.thickness, _dp(m.coords), m.ncell,
                                        _p(m.cells, c_int64_p), self.model, _dp(self.params.arr), _dp(ddu),
                                        _dp(self.sig), _dp(self.ivs), _p(self.elastic, c_uint8_p), self.nthreads,
                                        _p(bc, c_int64_p), _p(bi, c_int_p))
        if st == 2:
            raise OracleError("von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)", st,
                              int(bc[0]), int(bi[0]))
        if st:
            raise OracleError(f"update_secondary error {st} at cell {bc[0]} ip {bi[0]}", st, int(bc[0]), int(bi[0]))


def coo_to_csr(nrow, rows, cols, vals):
    """Sums duplicates in insertion order; returns (indptr, indices, data) as int64/int64/f64."""
    indptr = np.zeros(nrow + 1, np.int64)
    nnz = lib().orc_coo_to_csr(nrow, rows.size, _p(rows, c_int64_p), _p(cols, c_int64_p), _dp(vals),
                               _p(indptr, c_int64_p), None, None)
    indices = np.zeros(nnz, np.int64)
    data = np.zeros(nnz)
    lib().orc_coo_to_csr(nrow, rows.size, _p(rows, c_int64_p), _p(cols, c_int64_p), _dp(vals),
                         _p(indptr, c_int64_p), _p(indices, c_int64_p), _dp(data))
    return indptr, indices, data
