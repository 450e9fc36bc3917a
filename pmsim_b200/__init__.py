"""pmsim_b200 -- B200 (sm_100a) implementation of pmsim's implicit solid hot path.

* :mod:`pmsim_b200.elements` -- ``Elements``/``ElementTrait`` mirror (fused FP64 kernels, CSR gather)
* :mod:`pmsim_b200.material` -- batched von Mises return map + consistent tangent
* :mod:`pmsim_b200.solver`   -- ``SolverImplicit`` mirror (Newton/time loop)
* :mod:`pmsim_b200.mesh`     -- mesh container and structured generators
The compute path is ``libpms_b200.so`` (C ABI in include/pms.h); there is no CPU fallback.
"""
from .mesh import Mesh, structured_2d, structured_3d, read_msh  # noqa: F401
from .mesh import TRI3, TRI6, QUA4, QUA8, QUA9, TET4, TET10, HEX8, HEX20  # noqa: F401

__version__ = "0.1.0"


def load_library():
    from . import _lib

    return _lib.load()
