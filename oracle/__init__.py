"""CPU oracle for the gpu_mm pointing-operator hot path -- TEST INFRASTRUCTURE ONLY.

This package is the checker for the CUDA product path.  Only ``tests/``, ``__graft_entry__.smoke()``
and ``bench.py``'s CPU-baseline / reference legs may import it, and only to check or to time the CPU
baseline; the product (``gpu_mm_b200``) never imports it and has no CPU fallback.

Two native libraries sit behind it:

* ``liboracle.so`` -- the C restatement in ``oracle.c`` (every function cites the reference file:line
  it follows: ``map2tod_reference.cu``, ``tod2map_reference.cu``, ``gpu_mm_internals.hpp``,
  ``PointingPrePlan.cu``, ``PointingPlan.cu``, ``PointingPlanTester.cu``).
* ``_ref/libgpu_mm_ref.so`` (optional) -- the reference's own ``include/gpu_mm_internals.hpp``
  templates compiled from the reference source tree by ``oracle/Makefile``.  It pins the C
  restatement and serves as the "reference" CPU baseline.  It is built only where the reference
  tree exists; the committed golden vectors under ``tests/golden/`` carry its outputs elsewhere.
* ``_ref/libgpu_mm_refgpu.so`` (optional) -- the reference's own plan builder and planned /
  unplanned GPU operators (its ``src_lib`` sources, unchanged) compiled for sm_100a against a minimal
  stand-in for the ksgpu containers (``oracle/ksgpu_shim``).  It pins this implementation's plans to
  the reference's PointingPlan and PointingPlanTester and times the reference's kernels on the same
  GPU (``RefGpuPlan``, ``refgpu_*``).
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

ERR_BAD_YPIX = 0x1
ERR_BAD_XPIX = 0x2
ERR_INCONSISTENT_NMT = 0x4
ERR_NOT_IN_PIXELIZATION = 0x8


class LpixStruct(ctypes.Structure):
    _fields_ = [
        ("nypix_global", ctypes.c_int32),
        ("nxpix_global", ctypes.c_int32),
        ("periodic_xcoord", ctypes.c_int32),
        ("nycells", ctypes.c_int32),
        ("nxcells", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("ystride", ctypes.c_int64),
        ("polstride", ctypes.c_int64),
        ("cell_offsets", ctypes.POINTER(ctypes.c_int64)),
    ]


class Lpix:
    """Plain description of a local pixelization (gpu_mm.hpp:17-58) for the oracle."""

    def __init__(self, nypix_global, nxpix_global, cell_offsets, ystride, polstride, periodic_xcoord=True):
        self.cell_offsets = np.ascontiguousarray(cell_offsets, dtype=np.int64)
        assert self.cell_offsets.ndim == 2
        self.nypix_global = int(nypix_global)
        self.nxpix_global = int(nxpix_global)
        self.ystride = int(ystride)
        self.polstride = int(polstride)
        self.periodic_xcoord = bool(periodic_xcoord)
        self.nycells, self.nxcells = self.cell_offsets.shape
        self.npix = 64 * 64 * int(np.count_nonzero(self.cell_offsets >= 0))
        self.struct = LpixStruct(
            self.nypix_global, self.nxpix_global, int(self.periodic_xcoord), self.nycells, self.nxcells, 0,
            self.ystride, self.polstride, self.cell_offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))

    @classmethod
    def rectangle(cls, nypix_global, nxpix_global, periodic_xcoord=True):
        """Same layout as LocalPixelization.make_rectangle (gpu_mm.py:478-483)."""
        nyc = (nypix_global + 63) // 64
        nxc = (nxpix_global + 63) // 64
        offs = 64 * np.arange(nxc)[None, :] + 64 * 64 * nxc * np.arange(nyc)[:, None]
        return cls(nypix_global, nxpix_global, offs, 64 * nxc, 64 * 64 * nyc * nxc, periodic_xcoord)


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle: {path} is missing; run 'make -C oracle liboracle.so'")
        L = ctypes.CDLL(path)
        u32, i64, i32 = ctypes.c_uint32, ctypes.c_int64, ctypes.c_int32
        fp, dp = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        LP = ctypes.POINTER(LpixStruct)
        L.oracle_locate_f32.argtypes = [ctypes.c_float, ctypes.c_float, i32, i32, i32,
                                        ctypes.POINTER(i32), fp]
        L.oracle_locate_f32.restype = u32
        for name, T in (("f32", fp), ("f64", dp)):
            f = getattr(L, f"oracle_map2tod_{name}")
            f.argtypes = [T, T, T, i64, LP, i32, i32]
            f.restype = u32
            f = getattr(L, f"oracle_tod2map_{name}")
            f.argtypes = [T, T, T, i64, LP, i32]
            f.restype = u32
        L.oracle_response_map2tod_f32.argtypes = [fp, fp, fp, fp, i64, i64, LP, i32, i32]
        L.oracle_response_map2tod_f32.restype = u32
        L.oracle_response_tod2map_f32.argtypes = [fp, fp, fp, fp, i64, i64, LP, i32]
        L.oracle_response_tod2map_f32.restype = u32
        L.oracle_map2tod_f32_mt.argtypes = [fp, fp, fp, i64, LP, i32, i32, i32]
        L.oracle_map2tod_f32_mt.restype = u32
        L.oracle_tod2map_f32_mt.argtypes = [fp, fp, fp, i64, i64, LP, i32, i32]
        L.oracle_tod2map_f32_mt.restype = u32
        L.oracle_tod2map_f64w_mt.argtypes = [ctypes.POINTER(ctypes.c_double), fp, fp, i64, i64, LP, i32, i32]
        L.oracle_tod2map_f64w_mt.restype = u32
        L.oracle_preplan.argtypes = [fp, i64, i32, i32, i32, ctypes.POINTER(u32), ctypes.POINTER(i64),
                                     ctypes.POINTER(u32)]
        L.oracle_preplan.restype = i64
        L.oracle_plan.argtypes = [fp, i64, i32, i32, i32, i64, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(u32)]
        L.oracle_plan.restype = u32
        L.oracle_sample_slots.argtypes = [fp, i64, i32, i32, i32, ctypes.POINTER(i32)]
        L.oracle_line_counts.argtypes = [fp, i64, i32, i32, i32, ctypes.POINTER(ctypes.c_uint8)]
        _LIB = L
    return _LIB


def ref_path():
    return os.path.join(_HERE, "_ref", "libgpu_mm_ref.so")


def ref_available():
    return os.path.exists(ref_path())


def ref():
    """The reference-header build (oracle/_ref).  Raises if it was not built."""
    global _REF
    if _REF is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref was not built (it needs the reference source tree)")
        R = ctypes.CDLL(ref_path())
        u32, i64, i32 = ctypes.c_uint32, ctypes.c_int64, ctypes.c_int32
        fp, dp = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
        LP = ctypes.POINTER(LpixStruct)
        R.ref_locate_f32.argtypes = [ctypes.c_float, ctypes.c_float, i32, i32, i32, ctypes.POINTER(i32), fp]
        R.ref_locate_f32.restype = u32
        for name, T in (("f32", fp), ("f64", dp)):
            f = getattr(R, f"ref_map2tod_{name}")
            f.argtypes = [T, T, T, i64, LP, i32, i32]
            f.restype = u32
            f = getattr(R, f"ref_tod2map_{name}")
            f.argtypes = [T, T, T, i64, LP, i32]
            f.restype = u32
        R.ref_map2tod_f32_mt.argtypes = [fp, fp, fp, i64, LP, i32, i32, i32]
        R.ref_map2tod_f32_mt.restype = u32
        R.ref_tod2map_f32_mt.argtypes = [fp, fp, fp, i64, i64, LP, i32, i32]
        R.ref_tod2map_f32_mt.restype = u32
        R.ref_enumerate_gpu.argtypes = [ctypes.c_void_p, i64, i32, i32, i32, ctypes.c_void_p, ctypes.c_void_p]
        R.ref_enumerate_gpu.restype = i32
        _REF = R
    return _REF


def refgpu_path():
    return os.path.join(_HERE, "_ref", "libgpu_mm_refgpu.so")


def refgpu_available():
    return os.path.exists(refgpu_path())


_REFGPU = None


def refgpu():
    """The reference's own plan builder and GPU operators (oracle/_ref/libgpu_mm_refgpu.so: its
    src_lib sources compiled unchanged for sm_100a against oracle/ksgpu_shim).  Raises if it was not
    built."""
    global _REFGPU
    if _REFGPU is None:
        if not refgpu_available():
            raise RuntimeError("oracle/_ref/libgpu_mm_refgpu.so was not built (it needs the reference source tree)")
        R = ctypes.CDLL(refgpu_path())
        vp, l, i = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
        R.refgpu_last_error.restype = ctypes.c_char_p
        R.refgpu_plan_create.argtypes = [vp, l, l, l, i]
        R.refgpu_plan_create.restype = vp
        R.refgpu_plan_free.argtypes = [vp]
        R.refgpu_plan_info.argtypes = [vp, vp, vp]
        R.refgpu_plan_get.argtypes = [vp, vp, vp]
        R.refgpu_plan_tester.argtypes = [vp, l, l, l, i, vp, l, vp, vp]
        lp_args = [l, l, vp, vp, l, l, l, l, i]
        R.refgpu_planned_map2tod.argtypes = [vp, vp, vp, l, vp, l] + lp_args + [i, i]
        R.refgpu_planned_tod2map.argtypes = [vp, vp, l, vp, vp, l] + lp_args + [i]
        R.refgpu_unplanned_map2tod.argtypes = [vp, vp, l, vp, l] + lp_args + [vp, l, i, i]
        R.refgpu_unplanned_tod2map.argtypes = [vp, l, vp, vp, l] + lp_args + [vp, l, i]
        R.refgpu_reference_map2tod.argtypes = [vp, vp, l, vp, l, l, l, vp, l, l, l, l, i, i, i]
        R.refgpu_reference_tod2map.argtypes = [vp, l, vp, vp, l, l, l, vp, l, l, l, l, i, i]
        for name in ("plan_info", "plan_get", "plan_tester", "planned_map2tod", "planned_tod2map",
                     "unplanned_map2tod", "unplanned_tod2map", "reference_map2tod", "reference_tod2map"):
            getattr(R, "refgpu_" + name).restype = i
        _REFGPU = R
    return _REFGPU


def _refgpu_check(rc):
    if rc != 0:
        raise RuntimeError("reference: " + refgpu().refgpu_last_error().decode())


class RefGpuPlan:
    """PointingPrePlan + PointingPlan built by the reference's own code on the GPU.  'xp_gpu' is any
    (3, nsamp) float32 CUDA array with a data pointer (a torch tensor); the plan keeps no reference to
    it.  Device-array arguments of the methods are likewise raw CUDA tensors."""

    def __init__(self, xp_gpu, nypix_global, nxpix_global, periodic_xcoord=True):
        R = refgpu()
        self.nsamp = xp_gpu.numel() // 3
        self.ny, self.nx, self.periodic = int(nypix_global), int(nxpix_global), bool(periodic_xcoord)
        self.h = R.refgpu_plan_create(xp_gpu.data_ptr(), self.nsamp, self.ny, self.nx, int(self.periodic))
        if not self.h:
            raise RuntimeError("reference: " + R.refgpu_last_error().decode())
        info = np.zeros(8, np.int64)
        ov = ctypes.c_double()
        R.refgpu_plan_info(self.h, info.ctypes.data, ctypes.addressof(ov))
        (self.plan_nmt, self.ncl_per_threadblock, self.planner_nblocks, self.nmt_per_threadblock,
         self.pointing_nblocks, self.plan_nbytes, self.plan_constructor_tmp_nbytes, self.cub_nbytes) = \
            (int(v) for v in info)
        self.overhead = ov.value

    def __del__(self):
        if getattr(self, "h", None):
            refgpu().refgpu_plan_free(self.h)
            self.h = None

    def get(self):
        """(plan_mt uint64[plan_nmt] in the reference's own order, nmt_cumsum uint32[planner_nblocks])."""
        mt = np.zeros(self.plan_nmt, np.uint64)
        cs = np.zeros(1024, np.uint32)
        _refgpu_check(refgpu().refgpu_plan_get(self.h, mt.ctypes.data, cs.ctypes.data))
        return mt, cs[:self.planner_nblocks]

    @staticmethod
    def _lp(lp, offs_gpu):
        offs = np.ascontiguousarray(lp.cell_offsets, dtype=np.int64)
        return offs, [lp.nypix_global, lp.nxpix_global, offs.ctypes.data, offs_gpu.data_ptr(), lp.nycells,
                      lp.nxcells, lp.ystride, lp.polstride, int(lp.periodic_xcoord)]

    def map2tod(self, tod, lmap, xp, lp, offs_gpu, partial=False, accum=False):
        offs, a = self._lp(lp, offs_gpu)
        _refgpu_check(refgpu().refgpu_planned_map2tod(self.h, tod.data_ptr(), lmap.data_ptr(), lmap.numel(),
                                                      xp.data_ptr(), self.nsamp, *a, int(partial), int(accum)))

    def tod2map(self, lmap, tod, xp, lp, offs_gpu, partial=False):
        offs, a = self._lp(lp, offs_gpu)
        _refgpu_check(refgpu().refgpu_planned_tod2map(self.h, lmap.data_ptr(), lmap.numel(), tod.data_ptr(),
                                                      xp.data_ptr(), self.nsamp, *a, int(partial)))


def refgpu_unplanned_map2tod(tod, lmap, xp, lp, offs_gpu, errflags, partial=False, accum=False):
    offs, a = RefGpuPlan._lp(lp, offs_gpu)
    _refgpu_check(refgpu().refgpu_unplanned_map2tod(tod.data_ptr(), lmap.data_ptr(), lmap.numel(), xp.data_ptr(),
                                                    xp.numel() // 3, *a, errflags.data_ptr(), errflags.numel(),
                                                    int(partial), int(accum)))


def refgpu_unplanned_tod2map(lmap, tod, xp, lp, offs_gpu, errflags, partial=False):
    offs, a = RefGpuPlan._lp(lp, offs_gpu)
    _refgpu_check(refgpu().refgpu_unplanned_tod2map(lmap.data_ptr(), lmap.numel(), tod.data_ptr(), xp.data_ptr(),
                                                    xp.numel() // 3, *a, errflags.data_ptr(), errflags.numel(),
                                                    int(partial)))


def refgpu_plan_tester(xp_gpu, nypix_global, nxpix_global, periodic_xcoord=True, capacity=None):
    """The reference's PointingPlanTester (PointingPlanTester.cu:69-161): (sorted_mt, nmt_cumsum).
    'capacity' (at least the plan's nmt) sizes the output; by default 4 words per cache line."""
    nsamp = xp_gpu.numel() // 3
    cap = int(capacity) if capacity else 4 * (nsamp // 32) + 64
    mt = np.zeros(cap, np.uint64)
    cs = np.zeros(1024, np.uint32)
    n = ctypes.c_long()
    _refgpu_check(refgpu().refgpu_plan_tester(xp_gpu.data_ptr(), nsamp, int(nypix_global), int(nxpix_global),
                                              int(periodic_xcoord), mt.ctypes.data, cap, cs.ctypes.data,
                                              ctypes.addressof(n)))
    return mt[:n.value], cs


# ------------------------------------------------------------------------------------------------


def _nsamp(xpointing):
    xp = np.asarray(xpointing)
    assert xp.shape[0] == 3
    return xp.size // 3


def _ftype(dtype):
    return (ctypes.c_float, "f32") if np.dtype(dtype) == np.float32 else (ctypes.c_double, "f64")


def map2tod(tod, lmap, xpointing, lpix, partial_pixelization=False, accum=False, use_ref=False):
    """reference_map2tod semantics (map2tod_reference.cu:16-54).  Updates 'tod' in place and
    returns the error bits (bit 8 not masked)."""
    assert tod.flags["C_CONTIGUOUS"] and lmap.flags["C_CONTIGUOUS"] and xpointing.flags["C_CONTIGUOUS"]
    assert tod.dtype == lmap.dtype == xpointing.dtype
    ct, name = _ftype(tod.dtype)
    L = ref() if use_ref else lib()
    f = getattr(L, ("ref_map2tod_" if use_ref else "oracle_map2tod_") + name)
    return f(_ptr(tod, ct), _ptr(lmap, ct), _ptr(xpointing, ct), _nsamp(xpointing),
             ctypes.byref(lpix.struct), int(partial_pixelization), int(accum))


def tod2map(lmap, tod, xpointing, lpix, partial_pixelization=False, use_ref=False):
    """reference_tod2map semantics (tod2map_reference.cu:14-46): accumulates into 'lmap'."""
    assert tod.flags["C_CONTIGUOUS"] and lmap.flags["C_CONTIGUOUS"] and xpointing.flags["C_CONTIGUOUS"]
    assert tod.dtype == lmap.dtype == xpointing.dtype
    ct, name = _ftype(tod.dtype)
    L = ref() if use_ref else lib()
    f = getattr(L, ("ref_tod2map_" if use_ref else "oracle_tod2map_") + name)
    return f(_ptr(lmap, ct), _ptr(tod, ct), _ptr(xpointing, ct), _nsamp(xpointing),
             ctypes.byref(lpix.struct), int(partial_pixelization))


def map2tod_mt(tod, lmap, xpointing, lpix, nthreads, partial_pixelization=False, accum=False, use_ref=False):
    ct = ctypes.c_float
    f = ref().ref_map2tod_f32_mt if use_ref else lib().oracle_map2tod_f32_mt
    return f(_ptr(tod, ct), _ptr(lmap, ct), _ptr(xpointing, ct), _nsamp(xpointing), ctypes.byref(lpix.struct),
             int(partial_pixelization), int(accum), int(nthreads))


def tod2map_mt(lmap, tod, xpointing, lpix, nthreads, partial_pixelization=False, use_ref=False):
    ct = ctypes.c_float
    f = ref().ref_tod2map_f32_mt if use_ref else lib().oracle_tod2map_f32_mt
    return f(_ptr(lmap, ct), _ptr(tod, ct), _ptr(xpointing, ct), _nsamp(xpointing), lmap.size,
             ctypes.byref(lpix.struct), int(partial_pixelization), int(nthreads))


def tod2map_f64w_mt(lmap64, tod, xpointing, lpix, nthreads, partial_pixelization=False):
    """reference_tod2map<double> on float32 tod/xpointing widened to double; lmap64 is float64 and
    accumulates (the FP64 oracle of the tod2map precision variants)."""
    assert lmap64.dtype == np.float64 and tod.dtype == np.float32 and xpointing.dtype == np.float32
    return lib().oracle_tod2map_f64w_mt(_ptr(lmap64, ctypes.c_double), _ptr(tod, ctypes.c_float),
                                        _ptr(xpointing, ctypes.c_float), _nsamp(xpointing), lmap64.size,
                                        ctypes.byref(lpix.struct), int(partial_pixelization), int(nthreads))


def response_map2tod(tod, lmap, xpointing, response, lpix, partial_pixelization=False, accum=False):
    ndet = response.shape[1]
    nsamp = _nsamp(xpointing)
    ct = ctypes.c_float
    return lib().oracle_response_map2tod_f32(
        _ptr(tod, ct), _ptr(lmap, ct), _ptr(xpointing, ct), _ptr(np.ascontiguousarray(response), ct),
        ndet, nsamp // ndet, ctypes.byref(lpix.struct), int(partial_pixelization), int(accum))


def response_tod2map(lmap, tod, xpointing, response, lpix, partial_pixelization=False):
    ndet = response.shape[1]
    nsamp = _nsamp(xpointing)
    ct = ctypes.c_float
    return lib().oracle_response_tod2map_f32(
        _ptr(lmap, ct), _ptr(tod, ct), _ptr(xpointing, ct), _ptr(np.ascontiguousarray(response), ct),
        ndet, nsamp // ndet, ctypes.byref(lpix.struct), int(partial_pixelization))


def locate(y, x, ny, nx, periodic, use_ref=False):
    idx = (ctypes.c_int32 * 4)()
    d = (ctypes.c_float * 2)()
    f = ref().ref_locate_f32 if use_ref else lib().oracle_locate_f32
    err = f(float(y), float(x), int(ny), int(nx), int(periodic), idx, d)
    return tuple(idx), (np.float32(d[0]), np.float32(d[1])), err


def preplan(xpointing, nypix_global, nxpix_global, periodic_xcoord=True):
    """Returns dict(nmt, nmt_cumsum[1024], ncl_per_threadblock, planner_nblocks,
    nmt_per_threadblock, pointing_nblocks, err)  (PointingPrePlan.cu:129-251)."""
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    cum = np.zeros(1024, dtype=np.uint32)
    geom = np.zeros(4, dtype=np.int64)
    err = np.zeros(1, dtype=np.uint32)
    nmt = lib().oracle_preplan(_ptr(xp, ctypes.c_float), _nsamp(xp), int(nypix_global), int(nxpix_global),
                               int(periodic_xcoord), _ptr(cum, ctypes.c_uint32), _ptr(geom, ctypes.c_int64),
                               _ptr(err, ctypes.c_uint32))
    return dict(nmt=int(nmt), nmt_cumsum=cum, ncl_per_threadblock=int(geom[0]), planner_nblocks=int(geom[1]),
                nmt_per_threadblock=int(geom[2]), pointing_nblocks=int(geom[3]), err=int(err[0]))


def plan(xpointing, nypix_global, nxpix_global, periodic_xcoord=True, nmt=None):
    """Canonical plan: (plan_mt uint64[nmt] sorted by (cell, cache line) with exact mflag/zflag,
    owner_bits uint32[ceil(nmt/32)], err)."""
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    if nmt is None:
        nmt = preplan(xp, nypix_global, nxpix_global, periodic_xcoord)["nmt"]
    mt = np.zeros(max(nmt, 1), dtype=np.uint64)
    owner = np.zeros(max((nmt + 31) // 32, 1), dtype=np.uint32)
    err = lib().oracle_plan(_ptr(xp, ctypes.c_float), _nsamp(xp), int(nypix_global), int(nxpix_global),
                            int(periodic_xcoord), int(nmt), _ptr(mt, ctypes.c_uint64), _ptr(owner, ctypes.c_uint32))
    return mt[:nmt], owner[:(nmt + 31) // 32], int(err)


def owner_words(xpointing, nypix_global, mt, owner_bits):
    """Owner list of a single-TOD plan as the plan builder must produce it (the owner list is this
    implementation's own addition to the reference's plan; there is no reference counterpart).

    One word per cache line: the line's lowest cell | line << 20 | mflag << 46 | band << 48, sorted
    stably by (cell, band), i.e. in (cell, band, line) order.  'mt' and 'owner_bits' are plan()'s
    outputs (the owner bit marks the first mt word of each line in (cell, line) order, which is the
    line's lowest cell).  The band is the lowest upper bilinear row of the line's samples (locate's
    clamp of trunc(y) to [0, ny-2]) minus 64 * iycell of the owner, clamped to [0, 63]."""
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    n = _nsamp(xp)
    mt = np.asarray(mt, dtype=np.uint64)
    bits = np.unpackbits(np.asarray(owner_bits).view(np.uint8), bitorder="little")[:len(mt)].astype(bool)
    words = mt[bits] & np.uint64((1 << 47) - 1)          # cell, line, mflag (no zflag)
    lines = ((words >> np.uint64(20)) & np.uint64((1 << 26) - 1)).astype(np.int64)
    y = xp.reshape(3, n)[0][32 * lines[:, None] + np.arange(32)[None, :]].astype(np.float64)
    y = np.nan_to_num(y, nan=0.0, posinf=float(nypix_global), neginf=-1.0)
    iy0 = np.clip(np.trunc(np.clip(y, -1.0, float(nypix_global))), 0, nypix_global - 2).astype(np.int64).min(axis=1)
    iyc = ((words >> np.uint64(10)) & np.uint64(1023)).astype(np.int64)
    band = np.clip(iy0 - 64 * iyc, 0, 63).astype(np.uint64)
    words = words | (band << np.uint64(48))
    order = np.lexsort((lines, band, (words & np.uint64(0xFFFFF)).astype(np.int64)))
    return words[order]


def band_words(xpointing, nypix_global, nxpix_global, periodic_xcoord, owner):
    """Band words of a single-TOD plan, one per entry of its owner list 'owner' (as owner_words()
    gives it), as the plan builder must produce them (this implementation's own addition to the plan;
    no reference counterpart).  Bits: 0-31 same column as the previous sample; 32-38 first column in
    scan order, relative to the owner cell's x0; 39-44 number of columns; 45 x increases; 46 the line
    takes the tod2map band path; 47 some column holds three or four consecutive samples; 48 the
    samples' upper rows are R0 and R0 + 1 (not R0 only).  Zero for lines off that path."""
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    n = _nsamp(xp)
    owner = np.asarray(owner, dtype=np.uint64)
    lines = ((owner >> np.uint64(20)) & np.uint64((1 << 26) - 1)).astype(np.int64)
    cell = (owner & np.uint64(0xFFFFF)).astype(np.int64)
    band = ((owner >> np.uint64(48)) & np.uint64(63)).astype(np.int64)
    R0 = (cell >> 10) * 64 + band
    x0 = (cell & 1023) * 64
    idx = 32 * lines[:, None] + np.arange(32)[None, :]
    y = xp.reshape(3, n)[0][idx]
    x = xp.reshape(3, n)[1][idx]
    dy = (y - R0[:, None].astype(np.float32)).astype(np.float32)
    xr = (x - x0[:, None].astype(np.float32)).astype(np.float32)
    x_hi = np.float32(nxpix_global if periodic_xcoord else nxpix_global - 2)
    # Range checks on the float bit patterns as unsigned integers, as the builder does: negative
    # values (-0.0 included) and NaN fail.
    bits = lambda v: np.ascontiguousarray(v, dtype=np.float32).view(np.uint32)
    two = (bits(dy) >= bits(np.float32(1.0))).any(axis=1)
    rmax = np.where(two, nypix_global - 3, nypix_global - 2)
    ok = ((R0 <= rmax)[:, None] & (bits(dy) < bits(np.float32(2.0))) & (bits(xr) < bits(np.float32(95.0)))
          & (bits(x) < bits(x_hi)))
    k = np.floor(np.where(ok, xr, np.float32(0))).astype(np.int64)
    dk = np.diff(k, axis=1)
    bit = np.uint64(1) << np.arange(1, 32, dtype=np.uint64)
    su = ((dk == 0) * bit).sum(axis=1, dtype=np.uint64)
    up = ((dk == 1) * bit).sum(axis=1, dtype=np.uint64)
    down = ((dk == -1) * bit).sum(axis=1, dtype=np.uint64)
    r3 = su & (su >> np.uint64(1))
    fast = (ok.all(axis=1) & ((su | up | down) == np.uint64(0xFFFFFFFE)) & ~((up != 0) & (down != 0)) & (su != 0)
            & ((r3 & (r3 >> np.uint64(2))) == 0) & ~(two & (r3 != 0)))
    inc = down == 0
    kmin = np.where(inc, k[:, 0], k[:, 31])
    ncol = np.where(inc, k[:, 31], k[:, 0]) - kmin + 1
    w = (su | (kmin.astype(np.uint64) << np.uint64(32)) | (ncol.astype(np.uint64) << np.uint64(39))
         | (inc.astype(np.uint64) << np.uint64(45)) | (np.uint64(1) << np.uint64(46))
         | ((r3 != 0).astype(np.uint64) << np.uint64(47)) | (two.astype(np.uint64) << np.uint64(48)))
    return np.where(fast, w, np.uint64(0))


def sample_slots(xpointing, nypix_global, nxpix_global, periodic_xcoord=True):
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    n = _nsamp(xp)
    out = np.zeros(6 * n, dtype=np.int32)
    lib().oracle_sample_slots(_ptr(xp, ctypes.c_float), n, int(nypix_global), int(nxpix_global),
                              int(periodic_xcoord), _ptr(out, ctypes.c_int32))
    return out.reshape(n, 6)


def line_counts(xpointing, nypix_global, nxpix_global, periodic_xcoord=True):
    xp = np.ascontiguousarray(xpointing, dtype=np.float32)
    n = _nsamp(xp)
    out = np.zeros(n // 32, dtype=np.uint8)
    lib().oracle_line_counts(_ptr(xp, ctypes.c_float), n, int(nypix_global), int(nxpix_global),
                             int(periodic_xcoord), _ptr(out, ctypes.c_uint8))
    return out


def rel_l1(a, b):
    """The reference's comparison metric, sum|a-b| / (sum|a| + sum|b|)  (tests.py:220-224)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.abs(a).sum() + np.abs(b).sum()
    assert den > 0
    return float(np.abs(a - b).sum() / den)
