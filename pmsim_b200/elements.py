"""Host-side mirror of pmsim's ``Elements`` / ``ElementTrait`` for solids, on the B200 library.

Method names follow the reference (``src/fem/element_trait.rs:6-38``, ``src/fem/elements.rs:132-205``):
``initialize_internal_values``, ``reset_algorithmic_variables``, ``backup_secondary_values``,
``restore_secondary_values``, ``update_secondary_values``, ``assemble_f_int``, ``assemble_kk``,
``calc_f_int`` / ``calc_jacobian`` (one cell), plus the fused Newton call ``update_and_assemble``.
Each batched method is one C-ABI call (include/pms.h) over every cell; arrays may be numpy
(host, copied through) or CUDA tensors / raw device pointers (``device=True``).
Errors raise :class:`pmsim_b200._lib.PmsError` with the reference's message text.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .mesh import Mesh


class Material:
    """``StressStrain::VonMises {young, poisson, hh, z_ini}`` or ``LinearElastic {young, poisson}``."""

    def __init__(self, model="von_mises", young=1.0, poisson=0.0, hh=0.0, z_ini=1.0):
        self.model = _lib.VON_MISES if model in ("von_mises", _lib.VON_MISES) else _lib.LINEAR_ELASTIC
        self.young, self.poisson, self.hh, self.z_ini = float(young), float(poisson), float(hh), float(z_ini)

    def c(self):
        return _lib.material(self.model, self.young, self.poisson, self.hh, self.z_ini)

    @staticmethod
    def von_mises(young, poisson, hh, z_ini):
        return Material("von_mises", young, poisson, hh, z_ini)

    @staticmethod
    def linear_elastic(young, poisson):
        return Material("linear_elastic", young, poisson, 0.0, 1.0)


class Elements:
    def __init__(self, mesh: Mesh, materials, ngauss: int = 0, thickness: float = 1.0, cell_material=None,
                 axisymmetric: bool = False, plane_stress: bool = False):
        self.L = _lib.load()
        if isinstance(materials, Material):
            materials = [materials]
        self.mesh = mesh
        self.materials = list(materials)
        mats = (_lib.Material_ * len(materials))(*[m.c() for m in materials])
        self._cm = None
        if cell_material is not None:
            self._cm = np.ascontiguousarray(cell_material, dtype=np.int32)
        cmesh = _lib.Mesh_(mesh.ndim, mesh.kind, mesh.npoint, mesh.ncell, _lib.ptr(mesh.coords), _lib.ptr(mesh.cells),
                           _lib.ptr(self._cm))
        cfg = _lib.Config_(int(ngauss), 1 if plane_stress else 0, 1 if axisymmetric else 0, float(thickness))
        h = ctypes.c_void_p()
        rc = self.L.pms_elements_create(ctypes.byref(cmesh), mats, len(materials), ctypes.byref(cfg), ctypes.byref(h))
        if rc != _lib.PMS_OK:
            raw = self.L.pms_elements_last_error(None)  # the refusal's message (reference wording)
            raise _lib.PmsError(rc, raw.decode() if raw else None)
        self.h = h
        info = _lib.Info_()
        self.L.pms_elements_get_info(self.h, ctypes.byref(info))
        self.info = info
        self.ndim, self.ngauss, self.ncomp = info.ndim, info.ngauss, info.ncomp
        self.ndof, self.nip, self.nnz = info.ndof, info.nip, info.nnz
        self._pattern = None

    def close(self):
        if getattr(self, "h", None):
            self.L.pms_elements_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        _lib.check(rc, self.h)

    # ---- pattern --------------------------------------------------------------------------
    def csr_pattern(self):
        """(indptr int64[ndof+1], indices int32[nnz]) of K, columns sorted in each row."""
        if self._pattern is None:
            indptr = np.zeros(self.ndof + 1, np.int64)
            indices = np.zeros(self.nnz, np.int32)
            self._check(self.L.pms_elements_csr_pattern(self.h, _lib.ptr(indptr), _lib.ptr(indices),
                                                         _lib.PMS_MEM_HOST))
            self._pattern = (indptr, indices)
        return self._pattern

    def set_assembly(self, mode):
        """"gather" (default: upper element-matrix blocks, then row gathers summing every entry in
        ascending cell order) or "direct" (blocks added straight into the CSR values and R in the
        colour-major processing order); each reproducible, the two equal to the last bits."""
        code = {"direct": _lib.PMS_ASSEMBLY_DIRECT, "gather": _lib.PMS_ASSEMBLY_GATHER}[mode]
        self._check(self.L.pms_elements_set_assembly(self.h, code))

    def symmetric_jacobian(self):
        """ElementTrait::symmetric_jacobian (src/fem/element_solid.rs:100-102): True for the linear
        elastic and von Mises models."""
        out = ctypes.c_int32()
        self._check(self.L.pms_elements_symmetric_jacobian(self.h, ctypes.byref(out)))
        return bool(out.value)

    def set_symmetry(self, sym):
        """Storage of K in the CSR values, as russell_sparse's Sym (src/fem/linear_system.rs:119,
        src/base/assembly.rs:92-136): "full" (default, both triangles), "lower" (column <= row,
        Sym::YesLower) or "upper" (column >= row, Sym::YesUpper).  Changes ``nnz``,
        ``csr_pattern()`` and the values of ``assemble_kk`` / ``update_and_assemble``; the triangles
        need the gather assembly."""
        code = {"full": _lib.PMS_SYM_FULL, "lower": _lib.PMS_SYM_LOWER, "upper": _lib.PMS_SYM_UPPER}[sym]
        self._check(self.L.pms_elements_set_symmetry(self.h, code))
        info = _lib.Info_()
        self._check(self.L.pms_elements_get_info(self.h, ctypes.byref(info)))
        self.info, self.nnz = info, info.nnz
        self._pattern = None

    def set_stream(self, stream):
        """stream: torch.cuda.Stream, a raw cudaStream_t, or None for the handle's own stream."""
        raw = getattr(stream, "cuda_stream", stream)
        self._check(self.L.pms_elements_set_stream(self.h, raw))

    # ---- ElementTrait (batched) -------------------------------------------------------------
    def initialize_internal_values(self):
        self._check(self.L.pms_elements_initialize(self.h))

    def reset_algorithmic_variables(self):
        self._check(self.L.pms_elements_reset_algorithmic(self.h))

    def backup_secondary_values(self):
        self._check(self.L.pms_elements_backup(self.h))

    def restore_secondary_values(self):
        self._check(self.L.pms_elements_restore(self.h))

    def _mem(self, *arrays):
        dev = [a is not None and not isinstance(a, np.ndarray) for a in arrays]
        if any(dev) and not all(d for d, a in zip(dev, arrays) if a is not None):
            raise ValueError("mix of host and device buffers")
        return _lib.PMS_MEM_DEVICE if any(dev) else _lib.PMS_MEM_HOST

    @staticmethod
    def _host(a, n):
        if a is None:
            return None
        if isinstance(a, np.ndarray):
            a = np.ascontiguousarray(a, dtype=np.float64)
            if a.size < n:
                raise ValueError("array too short")
        return a

    def update_secondary_values(self, ddu):
        ddu = self._host(ddu, self.ndof)
        self._check(self.L.pms_elements_update_secondary(self.h, _lib.ptr(ddu), self._mem(ddu)))

    def assemble_f_int(self, out=None):
        if out is None:
            out = np.zeros(self.ndof)
        self._check(self.L.pms_elements_assemble_f_int(self.h, _lib.ptr(out), self._mem(out)))
        return out

    def assemble_kk(self, out=None):
        """CSR values of K in the order of ``csr_pattern()``."""
        if out is None:
            out = np.zeros(self.nnz)
        self._check(self.L.pms_elements_assemble_kk(self.h, _lib.ptr(out), self._mem(out)))
        return out

    def update_and_assemble(self, ddu, ff_int=None, csr_values=None):
        """restore + update_secondary_values(ddu) + assemble_f_int + assemble_kk in one pass.

        Starts every IP from the backed-up (step-start) state, as SolverImplicit::iterate does
        after backup (iteration 0) or restore (later iterations)."""
        ddu = self._host(ddu, self.ndof)
        self._check(self.L.pms_elements_update_and_assemble(self.h, _lib.ptr(ddu), _lib.ptr(ff_int),
                                                             _lib.ptr(csr_values),
                                                             self._mem(ddu, ff_int, csr_values)))
        return ff_int, csr_values

    def sync(self):
        self._check(self.L.pms_elements_sync(self.h))

    # ---- per cell -------------------------------------------------------------------------
    def calc_f_int(self, cell):
        f = np.zeros(self.mesh.nnode * self.ndim)
        self._check(self.L.pms_element_calc_f_int(self.h, int(cell), _lib.ptr(f)))
        return f

    def calc_jacobian(self, cell):
        ne = self.mesh.nnode * self.ndim
        k = np.zeros((ne, ne))
        self._check(self.L.pms_element_calc_jacobian(self.h, int(cell), _lib.ptr(k)))
        return k

    # ---- state ----------------------------------------------------------------------------
    def get_state(self):
        sig = np.zeros((self.nip, self.ncomp))
        ivs = np.zeros((self.nip, 2))
        el = np.zeros(self.nip, np.uint8)
        self._check(self.L.pms_elements_get_state(self.h, _lib.ptr(sig), _lib.ptr(ivs), _lib.ptr(el)))
        return sig, ivs, el

    def set_state(self, sig, ivs, elastic):
        sig = np.ascontiguousarray(sig, dtype=np.float64)
        ivs = np.ascontiguousarray(ivs, dtype=np.float64)
        el = np.ascontiguousarray(elastic, dtype=np.uint8)
        self._check(self.L.pms_elements_set_state(self.h, _lib.ptr(sig), _lib.ptr(ivs), _lib.ptr(el)))

    def launch_count(self):
        return int(self.L.pms_elements_launch_count(self.h))

    def error_location(self):
        c = ctypes.c_int64()
        i = ctypes.c_int32()
        self.L.pms_elements_error_location(self.h, ctypes.byref(c), ctypes.byref(i))
        return c.value, i.value
