"""ctypes binding of libpms_b200.so (declarations in include/pms.h).

The library is required: there is no CPU fallback.  If the shared object is missing this
module raises at load time with the build command to run.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpms_b200.so")

PMS_OK = 0
PMS_MEM_HOST = 0
PMS_MEM_DEVICE = 1
PMS_ERR_INVALID = 1
PMS_ERR_ZERO_SIGMA_D = 3
PMS_ERR_ZERO_NORM_S = 4
PMS_ERR_JACOBIAN = 5
PMS_ERR_UNSUPPORTED = 7
PMS_ERR_ORDER = 13
PMS_ASSEMBLY_DIRECT = 0
PMS_ASSEMBLY_GATHER = 1
PMS_SYM_FULL, PMS_SYM_LOWER, PMS_SYM_UPPER = 0, 1, 2
LINEAR_ELASTIC = 0
VON_MISES = 1

ERRORS = {
    1: "invalid argument",
    2: "CUDA runtime error",
    3: "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)",
    4: "von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)",
    5: "the determinant of the Jacobian must be positive",
    6: "out of device memory",
    7: "unsupported idealization or element kind",
    8: "batch too large for the fixed scratch of the no-allocation entry point",
    9: "cannot compute df/dsigma due to singularity",
    10: "plastic numerator (df/dsigma : De : deps) is overly negative",
    11: "the elastoplastic ODE took more than max_steps steps",
    12: "no yield-surface crossing found",
    13: "ordered assembly: a wait for an earlier cell timed out (internal error)",
}


class PmsError(RuntimeError):
    def __init__(self, code, msg=None):
        self.code = code
        super().__init__(msg or ERRORS.get(code, f"error {code}"))


class Mesh_(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int32), ("kind", ctypes.c_int32), ("npoint", ctypes.c_int64),
                ("ncell", ctypes.c_int64), ("coords", ctypes.c_void_p), ("cells", ctypes.c_void_p),
                ("cell_material", ctypes.c_void_p)]


class Material_(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("young", ctypes.c_double), ("poisson", ctypes.c_double),
                ("hh", ctypes.c_double), ("z_ini", ctypes.c_double)]


class Config_(ctypes.Structure):
    _fields_ = [("ngauss", ctypes.c_int32), ("plane_stress", ctypes.c_int32), ("axisymmetric", ctypes.c_int32),
                ("thickness", ctypes.c_double)]


class BatchConfig_(ctypes.Structure):
    _fields_ = [("tol_rr_abs", ctypes.c_double), ("tol_mdu_rel", ctypes.c_double),
                ("n_max_iterations", ctypes.c_int32), ("pcg_rtol", ctypes.c_double),
                ("pcg_max_iterations", ctypes.c_int32), ("constant_tangent", ctypes.c_int32)]


class BatchTuning_(ctypes.Structure):
    _fields_ = [("team_max_ndof", ctypes.c_int64), ("team_threads", ctypes.c_int32),
                ("team_chunks", ctypes.c_int32), ("pcg_budget", ctypes.c_int32), ("graph_iters", ctypes.c_int32)]


class EpSettings_(ctypes.Structure):
    _fields_ = [("tol_rel", ctypes.c_double), ("tol_abs", ctypes.c_double), ("h_ini", ctypes.c_double),
                ("max_steps", ctypes.c_int32), ("pad_", ctypes.c_int32)]


class Info_(ctypes.Structure):
    _fields_ = [("ndim", ctypes.c_int32), ("kind", ctypes.c_int32), ("nnode", ctypes.c_int32),
                ("ngauss", ctypes.c_int32), ("ncomp", ctypes.c_int32), ("npoint", ctypes.c_int64),
                ("ncell", ctypes.c_int64), ("ndof", ctypes.c_int64), ("nip", ctypes.c_int64),
                ("nnz", ctypes.c_int64), ("nblock_upper", ctypes.c_int64), ("ncontrib", ctypes.c_int64),
                ("device_bytes", ctypes.c_int64)]


# every exported symbol and its (restype, argtypes); the CPU test checks this list against pms.h
_V, _I, _I64, _D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "pms_elements_create": (_I, [ctypes.POINTER(Mesh_), ctypes.POINTER(Material_), _I, ctypes.POINTER(Config_),
                                 ctypes.POINTER(_V)]),
    "pms_elements_destroy": (None, [_V]),
    "pms_elements_get_info": (_I, [_V, ctypes.POINTER(Info_)]),
    "pms_elements_set_stream": (_I, [_V, _V]),
    "pms_elements_csr_pattern": (_I, [_V, _V, _V, _I]),
    "pms_elements_initialize": (_I, [_V]),
    "pms_elements_reset_algorithmic": (_I, [_V]),
    "pms_elements_backup": (_I, [_V]),
    "pms_elements_restore": (_I, [_V]),
    "pms_elements_update_secondary": (_I, [_V, _V, _I]),
    "pms_elements_assemble_f_int": (_I, [_V, _V, _I]),
    "pms_elements_assemble_kk": (_I, [_V, _V, _I]),
    "pms_elements_update_and_assemble": (_I, [_V, _V, _V, _V, _I]),
    "pms_element_calc_f_int": (_I, [_V, _I64, _V]),
    "pms_element_calc_jacobian": (_I, [_V, _I64, _V]),
    "pms_elements_get_state": (_I, [_V, _V, _V, _V]),
    "pms_elements_set_state": (_I, [_V, _V, _V, _V]),
    "pms_elements_sync": (_I, [_V]),
    "pms_elements_last_error": (ctypes.c_char_p, [_V]),
    "pms_elements_error_location": (_I, [_V, ctypes.POINTER(_I64), ctypes.POINTER(_I)]),
    "pms_elements_launch_count": (_I64, [_V]),
    "pms_vm_update_and_stiffness_batch": (_I, [ctypes.POINTER(Material_), _I, _I64, _V, _V, _V, _V, _V, _V, _V,
                                               _V, _V]),
    "pms_vm_stiffness_batch": (_I, [ctypes.POINTER(Material_), _I, _I64, _V, _V, _V, _V, _V, _V, _V]),
    "pms_ep_update_stress_batch": (_I, [ctypes.POINTER(Material_), _I, _I64, _V, _V, _V, _V,
                                        ctypes.POINTER(EpSettings_), _V, _V, _V, _V]),
    "pms_ep_update_stress_host": (_I, [ctypes.POINTER(Material_), _I, _I64, _V, _V, _V, _V,
                                       ctypes.POINTER(EpSettings_), _V, _V]),
    "pms_vm_update_and_stiffness_host": (_I, [ctypes.POINTER(Material_), _I, _I64, _V, _V, _V, _V, _V, _V, _V]),
    "pms_mesh_csr_pattern": (_I, [ctypes.POINTER(Mesh_), _V, _V, ctypes.POINTER(_I64)]),
    "pms_mesh_csr_pattern_sym": (_I, [ctypes.POINTER(Mesh_), _I, _V, _V, ctypes.POINTER(_I64)]),
    "pms_elements_set_timing": (_I, [_V, _I]),
    "pms_elements_set_assembly": (_I, [_V, _I]),
    "pms_elements_set_symmetry": (_I, [_V, _I]),
    "pms_elements_symmetric_jacobian": (_I, [_V, _V]),
    "pms_set_device": (_I, [_I]),
    "pms_shape_table": (_I, [_I, _I, _V, _V]),
    "pms_mesh_assembly_maps": (_I, [ctypes.POINTER(Mesh_), _V, _V, _V, _V]),
    "pms_device_count": (_I, [_V]),
    "pms_elements_kernel_times": (_I, [_V, _V, _V]),
    "pms_probe_fp64_fma": (_I, [_I64, _I, _V, _V]),
    "pms_element_calc_noalloc": (_I, [_I, _I, _D, ctypes.POINTER(Material_), _I64, _V, _V, _V, _V, _V, _V,
                                      ctypes.POINTER(_I64), _V]),
    "pms_batch_create": (_I, [_V, _I, _V, _V, _I64, _V, _V, ctypes.POINTER(BatchConfig_), ctypes.POINTER(_V)]),
    "pms_batch_destroy": (None, [_V]),
    "pms_batch_reset": (_I, [_V]),
    "pms_batch_solve_step": (_I, [_V, _V, _V, _V, _V, _V, _V]),
    "pms_batch_tick": (_I, [_V, _V, _V, _V, _V, _V, _V]),
    "pms_batch_solve_step_graph": (_I, [_V, _V, _V, _V, _V, _V, _V]),
    "pms_batch_host_syncs": (_I64, [_V]),
    "pms_batch_set_tuning": (_I, [_V, ctypes.POINTER(BatchTuning_)]),
    "pms_batch_get_tuning": (_I, [_V, ctypes.POINTER(BatchTuning_)]),
    "pms_batch_autotune": (_I, [_V, ctypes.POINTER(BatchTuning_)]),
    "pms_batch_time_pcg": (_I, [_V, ctypes.POINTER(BatchTuning_), _I, ctypes.POINTER(_D)]),
    "pms_batch_get_u": (_I, [_V, _V]),
    "pms_batch_get_multipliers": (_I, [_V, _V]),
    "pms_batch_counters": (_I64, [_V, ctypes.POINTER(_I64)]),
    "pms_batch_last_error": (ctypes.c_char_p, [_V]),
    "pms_dpcg_create": (_I, [_I, _I64, _I64, _V, _V, _V, _I64, _V, _I64, _V, ctypes.POINTER(_V)]),
    "pms_dpcg_destroy": (None, [_V]),
    "pms_dpcg_last_error": (ctypes.c_char_p, [_V]),
    "pms_dpcg_set_stream": (_I, [_V, _V]),
    "pms_dpcg_bind": (_I, [_V, _V, _V, _V, _V, _V, _V, _V, _V]),
    "pms_dpcg_set_values": (_I, [_V, _V]),
    "pms_dpcg_start": (_I, [_V, _V]),
    "pms_dpcg_init": (_I, [_V]),
    "pms_dpcg_pack": (_I, [_V]),
    "pms_dpcg_unpack": (_I, [_V]),
    "pms_dpcg_spmv": (_I, [_V, _I]),
    "pms_dpcg_dot_pq": (_I, [_V]),
    "pms_dpcg_update": (_I, [_V]),
    "pms_dpcg_direction": (_I, [_V, _D]),
    "pms_dpcg_info": (_I, [_V, _V]),
    "pms_version": (ctypes.c_char_p, []),
    "pms_material_launch_count": (_I64, []),
}

_lib = None


def load(path: str | None = None):
    """Loads (once) and returns the library.  Raises if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m pmsim_b200.build` (nvcc, sm_100a)")
    L = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def material(model=VON_MISES, young=1.0, poisson=0.0, hh=0.0, z_ini=1.0) -> Material_:
    return Material_(int(model), float(young), float(poisson), float(hh), float(z_ini))


def ptr(a) -> int | None:
    """Address of a numpy array, a torch tensor or an int; None for None."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"cannot take the address of {type(a)}")


def check(code: int, handle=None):
    if code != PMS_OK:
        msg = None
        if handle is not None:
            raw = load().pms_elements_last_error(handle)
            msg = raw.decode() if raw else None
        raise PmsError(code, msg)


def set_device(device: int):
    """Makes `device` current for the calling host thread (handles then live on it)."""
    check(load().pms_set_device(int(device)))


def device_count() -> int:
    n = ctypes.c_int32(0)
    load().pms_device_count(ctypes.byref(n))
    return int(n.value)
