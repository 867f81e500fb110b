"""gpu_mm_b200: B200-native (sm_100a) pointing operators for CMB map-making, a drop-in for the
pointing-operator path of kmsmith137/gpu_mm (map2tod, tod2map, LocalPixelization, LocalMap,
DynamicMap, PointingPrePlan, PointingPlan).

Layers: hand-written CUDA kernels + C ABI (libgpu_mm_b200.so, include/gpu_mm_b200.h) -> C++ API
(include/gpu_mm_b200/gpu_mm.hpp) -> pybind11 module gpu_mm_pybind11 -> this package.
Build with ``python gpu_mm_b200/build.py``.  There is no CPU fallback: importing without the native
extension fails.
"""

import os as _os

_HERE = _os.path.dirname(_os.path.abspath(__file__))

try:
    from . import gpu_mm_pybind11
except ImportError as _e:   # pragma: no cover - exercised only on unbuilt trees
    raise ImportError(
        "gpu_mm_b200: native extension not built or not loadable "
        f"({_e}); run 'python gpu_mm_b200/build.py' (needs nvcc)") from _e

from .gpu_mm import *            # noqa: F401,F403
from .gpu_mm import (map2tod, tod2map, LocalPixelization, LocalMap, DynamicMap, PointingPrePlan,  # noqa: F401
                     PointingPlan, read_xpointing_npzfile, mm_dtype, ToyPointing, PointingPlanTester, tod2map_compensated, fold_compensation,
                     tod2map_f64, HotCells, tod2map_hot_f64)

from .batch import TodBatch  # noqa: E402,F401
from . import autotune  # noqa: E402,F401
from .serving import PointingServer  # noqa: E402,F401
from .host_pipeline import HostPipeline  # noqa: E402,F401

__all__ = ["map2tod", "tod2map", "LocalPixelization", "LocalMap", "DynamicMap", "PointingPrePlan",
           "PointingPlan", "read_xpointing_npzfile", "mm_dtype", "gpu_mm_pybind11", "tod2map_compensated",
           "fold_compensation", "tod2map_f64", "HotCells", "tod2map_hot_f64", "TodBatch", "autotune", "PointingServer"]


def library_path():
    """Path of the C-ABI shared library (libgpu_mm_b200.so)."""
    return _os.path.join(_HERE, "libgpu_mm_b200.so")
