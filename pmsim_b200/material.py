"""Batched ``StressStrainTrait`` calls for von Mises / linear elasticity on the B200 library.

``update_stress`` + ``stiffness`` of the reference (``src/material/von_mises.rs:124-226``,
``src/material/linear_elastic.rs:49-71``) run per IP behind a trait object; here one call
updates n IPs held as structure-of-arrays (component stride n):

    sig[ncomp, n] (Mandel), z[n], lambda[n], elastic[n] (uint8), deps[ncomp, n],
    dd[nd, n]: upper triangle (row-major, i <= j) of the Mandel tangent, nd = 21 (3D) / 10 (2D).

Device buffers are CUDA tensors (or raw pointers); host buffers are numpy arrays.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def upper_index(ncomp):
    """(i, j) of each stored tangent component, i <= j, row-major."""
    return [(i, j) for i in range(ncomp) for j in range(i, ncomp)]


def unpack_tangent(dd, ncomp):
    """dd[nd, n] -> D[n, ncomp, ncomp] (numpy)."""
    dd = np.asarray(dd)
    n = dd.shape[1]
    out = np.zeros((n, ncomp, ncomp))
    for k, (i, j) in enumerate(upper_index(ncomp)):
        out[:, i, j] = dd[k]
        out[:, j, i] = dd[k]
    return out


class VonMisesBatch:
    """StressStrain::VonMises {young, poisson, hh, z_ini} (model="linear_elastic" for Hooke)."""

    def __init__(self, young, poisson, hh=0.0, z_ini=1.0, ndim=3, model="von_mises"):
        self.L = _lib.load()
        m = _lib.VON_MISES if model == "von_mises" else _lib.LINEAR_ELASTIC
        self.mat = _lib.material(m, young, poisson, hh, z_ini)
        self.ndim = ndim
        self.ncomp = 2 * ndim
        self.ntan = self.ncomp * (self.ncomp + 1) // 2

    def update_and_stiffness(self, sig, z, lam, elastic, deps, hh=None, dd=None, status=None, stream=None):
        """Device call (tensors on cuda): in-place update of sig/z/lam/elastic, tangent into dd."""
        n = sig.shape[-1]
        raw = getattr(stream, "cuda_stream", stream)
        rc = self.L.pms_vm_update_and_stiffness_batch(ctypes.byref(self.mat), self.ndim, n, _lib.ptr(sig),
                                                      _lib.ptr(z), _lib.ptr(lam), _lib.ptr(elastic),
                                                      _lib.ptr(deps), _lib.ptr(hh), _lib.ptr(dd),
                                                      _lib.ptr(status), raw)
        _lib.check(rc)

    def stiffness(self, sig, lam, elastic, dd, hh=None, status=None, stream=None):
        n = sig.shape[-1]
        raw = getattr(stream, "cuda_stream", stream)
        rc = self.L.pms_vm_stiffness_batch(ctypes.byref(self.mat), self.ndim, n, _lib.ptr(sig), _lib.ptr(lam),
                                           _lib.ptr(elastic), _lib.ptr(hh), _lib.ptr(dd), _lib.ptr(status), raw)
        _lib.check(rc)

    def update_and_stiffness_host(self, sig, z, lam, elastic, deps, hh=None, with_tangent=True):
        """Host numpy buffers (copied to the device and back inside the call). Returns dd or None."""
        n = sig.shape[-1]
        for a in (sig, z, lam, elastic, deps):
            if not a.flags["C_CONTIGUOUS"]:
                raise ValueError("host arrays must be C-contiguous")
        dd = np.zeros((self.ntan, n)) if with_tangent else None
        rc = self.L.pms_vm_update_and_stiffness_host(ctypes.byref(self.mat), self.ndim, n, _lib.ptr(sig),
                                                     _lib.ptr(z), _lib.ptr(lam), _lib.ptr(elastic),
                                                     _lib.ptr(deps), _lib.ptr(hh), _lib.ptr(dd))
        _lib.check(rc)
        return dd


EP_CASES = ("AE", "AXB", "BE", "BXP", "BP")


class ElastoplasticBatch:
    """``Elastoplastic::update_stress`` (``src/material/elastoplastic.rs:539-641``) over n IPs.

    The general elastoplastic update of the reference with its one plasticity model, von Mises
    (``src/material/von_mises.rs:229-282``): the crossing of the yield surface along the elastic
    path, then the ODE ``dsigma/dt = Dep : deps``, ``dz/dt = Lambda_d H`` integrated (Dormand-Prince
    5(4), adaptive) from the crossing to the end of the increment.  Device buffers, structure of
    arrays: sig[ncomp, n], z[n], elastic[n] (uint8) updated in place from deps[ncomp, n]; cases[n]
    (int32, optional) receives the index into ``EP_CASES`` (-1 where the IP failed) and steps[n]
    the ODE steps.  There is no tangent, as in the reference (``Elastoplastic::stiffness`` is a
    TODO there).
    """

    def __init__(self, young, poisson, hh, z_ini, ndim=3, tol_rel=1e-10, tol_abs=1e-10, h_ini=1.0,
                 max_steps=1000):
        self.L = _lib.load()
        self.mat = _lib.material(_lib.VON_MISES, young, poisson, hh, z_ini)
        self.ndim = ndim
        self.ncomp = 2 * ndim
        self.settings = _lib.EpSettings_(tol_rel, tol_abs, h_ini, max_steps, 0)

    def update_stress(self, sig, z, elastic, deps, cases=None, steps=None, status=None, stream=None):
        n = sig.shape[-1]
        raw = getattr(stream, "cuda_stream", stream)
        rc = self.L.pms_ep_update_stress_batch(ctypes.byref(self.mat), self.ndim, n, _lib.ptr(sig), _lib.ptr(z),
                                               _lib.ptr(elastic), _lib.ptr(deps), ctypes.byref(self.settings),
                                               _lib.ptr(cases), _lib.ptr(steps), _lib.ptr(status), raw)
        _lib.check(rc)

    def update_stress_host(self, sig, z, elastic, deps):
        """Host numpy buffers (SoA as above; copied to the device and back inside the call).
        Returns (code of the first failing IP or 0, cases, steps)."""
        n = sig.shape[-1]
        for a in (sig, z, elastic, deps):
            if not a.flags["C_CONTIGUOUS"]:
                raise ValueError("host arrays must be C-contiguous")
        cases = np.zeros(n, dtype=np.int32)
        steps = np.zeros(n, dtype=np.int32)
        rc = self.L.pms_ep_update_stress_host(ctypes.byref(self.mat), self.ndim, n, _lib.ptr(sig), _lib.ptr(z),
                                              _lib.ptr(elastic), _lib.ptr(deps), ctypes.byref(self.settings),
                                              _lib.ptr(cases), _lib.ptr(steps))
        if rc in (1, 2, 6):  # invalid argument, CUDA error, no device memory: not a per-IP outcome
            _lib.check(rc)
        return rc, cases, steps
