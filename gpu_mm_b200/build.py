"""Build recipe for the gpu_mm_b200 native libraries (in-tree, sm_100a).

Produces, next to this file:
  libgpu_mm_b200.so                        CUDA kernels + C ABI + C++ API (static cudart)
  gpu_mm_pybind11<EXT_SUFFIX>              pybind11 module linked against it (rpath $ORIGIN)

nvcc cross-compiles for sm_100a without a GPU, so this runs anywhere the CUDA toolkit is installed.
"""

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)

CU_SOURCES = ["plan_kernels.cu", "operator_kernels.cu", "cell_kernels.cu", "tod_kernels.cu", "f64_kernels.cu", "quantize_kernels.cu", "capi.cu", "noalloc.cu", "cpp_api.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libgpu_mm_b200.so")


def _nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if os.path.exists(cand) else "nvcc"


def _cuda_include():
    return os.path.join(os.path.dirname(os.path.dirname(_nvcc())), "include") if os.path.isabs(_nvcc()) \
        else "/usr/local/cuda/include"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ... (exit {r.returncode})")
    return r


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps += [os.path.join(ROOT, "include", "gpu_mm_b200.h"),
             os.path.join(ROOT, "include", "gpu_mm_b200", "gpu_mm.hpp"), __file__]
    return deps


def pyext_path():
    return os.path.join(HERE, "gpu_mm_pybind11" + sysconfig.get_config_var("EXT_SUFFIX"))


def build(verbose=False, force=False):
    deps = _deps()
    if force or not _newer(LIB, deps):
        cmd = [_nvcc(), "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3",
               "-shared", "-o", LIB] + [os.path.join(CSRC, f) for f in CU_SOURCES]
        _run(cmd, verbose)
    ext = pyext_path()
    if force or not _newer(ext, deps + [LIB]):
        import pybind11
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden",
               "-I" + sysconfig.get_paths()["include"], "-I" + pybind11.get_include(), "-I" + _cuda_include(),
               os.path.join(CSRC, "pybind_module.cpp"), "-L" + HERE, "-lgpu_mm_b200",
               "-Wl,-rpath,$ORIGIN", "-o", ext]
        _run(cmd, verbose)
    return LIB, ext


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
