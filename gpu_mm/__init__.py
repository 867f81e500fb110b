"""The import name of the reference's Python package (kmsmith137/gpu_mm), bound to this build.

Code written against the reference's pointing operators runs unchanged: ``import gpu_mm``,
``from gpu_mm import map2tod, PointingPlan, ...``, ``from gpu_mm import gpu_mm_pybind11``,
``import gpu_mm.gpu_mm_pybind11`` and ``from gpu_mm.gpu_mm import ...`` all resolve to
``gpu_mm_b200`` and its native module.  Only the pointing-operator path exists here: the reference's
cuFFT/cuBLAS helpers (gpu_utils, gpu_pointing, pycufft) and MPI pixelizations are not part of it.
"""

import sys as _sys

import gpu_mm_b200 as _impl
from gpu_mm_b200 import *  # noqa: F401,F403
from gpu_mm_b200 import gpu_mm_pybind11  # noqa: F401
from gpu_mm_b200 import gpu_mm  # noqa: F401  (the reference's gpu_mm/gpu_mm.py module)

_sys.modules[__name__ + ".gpu_mm_pybind11"] = _impl.gpu_mm_pybind11
_sys.modules[__name__ + ".gpu_mm"] = _impl.gpu_mm

__doc__ = (__doc__ or "") + "\n" + (_impl.gpu_mm.__doc__ or "")
