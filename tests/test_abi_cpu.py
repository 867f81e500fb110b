"""CPU checks of the drop-in boundary: the C-ABI library loads and exports every entry point that
include/gpu_mm_b200.h declares, host-side geometry equals the reference's, and argument validation
rejects bad calls before any device work.  No GPU is touched."""

import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from tests._common import random_raster

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class PreplanInfo(ctypes.Structure):
    _fields_ = [("nsamp", ctypes.c_int64), ("nypix_global", ctypes.c_int32), ("nxpix_global", ctypes.c_int32),
                ("periodic_xcoord", ctypes.c_int32), ("sort_digit_bits", ctypes.c_int32),
                ("plan_nbytes", ctypes.c_int64), ("plan_constructor_tmp_nbytes", ctypes.c_int64),
                ("overhead", ctypes.c_double), ("ncl_per_threadblock", ctypes.c_int64),
                ("planner_nblocks", ctypes.c_int64), ("nmt_per_threadblock", ctypes.c_int64),
                ("pointing_nblocks", ctypes.c_int64), ("plan_nmt", ctypes.c_int64), ("sort_nbytes", ctypes.c_int64)]


class PlanLayout(ctypes.Structure):
    _fields_ = [("mt_offset", ctypes.c_int64), ("err_offset", ctypes.c_int64), ("owner_offset", ctypes.c_int64),
                ("cellmap_offset", ctypes.c_int64), ("total_nbytes", ctypes.c_int64), ("band_offset", ctypes.c_int64)]


@pytest.fixture(scope="module")
def lib():
    path = os.path.join(ROOT, "gpu_mm_b200", "libgpu_mm_b200.so")
    if not os.path.exists(path):
        pytest.fail("libgpu_mm_b200.so is not built (run python gpu_mm_b200/build.py)")
    L = ctypes.CDLL(path)
    L.gmm_last_error.restype = ctypes.c_char_p
    L.gmm_version.restype = ctypes.c_char_p
    return L


def declared_symbols():
    hdrs = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
    names = set()
    for h in hdrs:
        text = open(h).read()
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(gmm_\w+)\s*\(", text, re.M))
    return sorted(names)


def test_every_declared_entry_point_is_exported(lib):
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/*.h but not exported"


def test_version_and_last_error(lib):
    assert b"sm_100a" in lib.gmm_version()
    assert lib.gmm_last_error() == b""


@pytest.mark.parametrize("nsamp_lines,nmt", [(1, 1), (700, 1900), (1024 * 16, 40000), (1 << 20, 3 << 20)])
def test_preplan_info_matches_reference_geometry(lib, nsamp_lines, nmt):
    info = PreplanInfo()
    rc = lib.gmm_preplan_info_init(ctypes.c_int64(32 * nsamp_lines), 1000, 2000, 1, ctypes.c_int64(nmt),
                                   ctypes.byref(info))
    assert rc == 0
    ncl = nsamp_lines
    c = max(16, -(-ncl // 1024))
    c = (c + 3) & ~3
    assert info.ncl_per_threadblock == c
    assert info.planner_nblocks == -(-ncl // c)
    npt = (int(np.sqrt(nmt)) + 32) & ~31
    assert info.nmt_per_threadblock == npt
    assert info.pointing_nblocks == -(-nmt // npt)
    assert info.plan_nmt == nmt
    assert abs(info.overhead - (32 * nmt / (32.0 * nsamp_lines) - 1.0)) < 1e-12
    lay = PlanLayout()
    assert lib.gmm_plan_layout_get(ctypes.byref(info), ctypes.byref(lay)) == 0
    assert lay.total_nbytes == info.plan_nbytes
    assert lay.err_offset >= 8 * nmt and lay.err_offset % 128 == 0 and lay.owner_offset % 128 == 0
    assert lay.cellmap_offset >= lay.owner_offset + 8 * nsamp_lines and lay.cellmap_offset % 128 == 0
    assert lay.band_offset - lay.cellmap_offset == (1 << 20) // 8 and lay.band_offset % 128 == 0
    assert lay.total_nbytes >= lay.band_offset + 8 * nsamp_lines


def test_preplan_geometry_matches_oracle(lib):
    rng = np.random.default_rng(1)
    xp = random_raster(rng, 3, 32 * 300, 120, 200, True)
    pp = oracle.preplan(xp, 120, 200, True)
    info = PreplanInfo()
    assert lib.gmm_preplan_info_init(ctypes.c_int64(xp.size // 3), 120, 200, 1, ctypes.c_int64(pp["nmt"]),
                                     ctypes.byref(info)) == 0
    for k in ("ncl_per_threadblock", "planner_nblocks", "nmt_per_threadblock", "pointing_nblocks"):
        assert getattr(info, k) == pp[k], k


def test_invalid_arguments_rejected_before_device_work(lib):
    info = PreplanInfo()
    # nsamp not a multiple of 32 (check_arguments.cu:20-25)
    rc = lib.gmm_preplan(ctypes.c_void_p(16), ctypes.c_int64(33), 100, 100, 1, ctypes.c_void_p(16),
                         ctypes.c_void_p(16), 0, None, ctypes.byref(info))
    assert rc == 0x100
    assert b"multiple of 32" in lib.gmm_last_error()
    # empty and oversized TODs: nsamp must be in [32, 2^31]
    for nsamp in (0, -32, (1 << 31) + 32):
        rc = lib.gmm_preplan(ctypes.c_void_p(16), ctypes.c_int64(nsamp), 100, 100, 1, ctypes.c_void_p(16),
                             ctypes.c_void_p(16), 0, None, ctypes.byref(info))
        assert rc == 0x100 and b"nsamp" in lib.gmm_last_error(), nsamp
    assert lib.gmm_preplan_info_init(ctypes.c_int64(1 << 31), 100, 100, 1, ctypes.c_int64(1 << 26),
                                     ctypes.byref(info)) == 0
    # map too large (check_arguments.cu:28-39)
    rc = lib.gmm_preplan(ctypes.c_void_p(16), ctypes.c_int64(64), 70000, 100, 1, ctypes.c_void_p(16),
                         ctypes.c_void_p(16), 0, None, ctypes.byref(info))
    assert rc == 0x100
    # null pointer
    rc = lib.gmm_preplan(None, ctypes.c_int64(64), 100, 100, 1, ctypes.c_void_p(16), ctypes.c_void_p(16), 0, None,
                         ctypes.byref(info))
    assert rc == 0x100 and b"xpointing" in lib.gmm_last_error()
    # plan buffers too small
    assert lib.gmm_preplan_info_init(ctypes.c_int64(64 * 32), 100, 100, 1, ctypes.c_int64(100), ctypes.byref(info)) == 0
    rc = lib.gmm_plan_build(ctypes.byref(info), ctypes.c_void_p(128), ctypes.c_void_p(128), ctypes.c_void_p(128),
                            ctypes.c_int64(16), ctypes.c_void_p(128), ctypes.c_int64(16), 0, None)
    assert rc == 0x400
    assert b"buf" in lib.gmm_last_error()
    # nmt out of range (PointingPrePlan.cu:213-214)
    assert lib.gmm_preplan_info_init(ctypes.c_int64(64), 100, 100, 1, ctypes.c_int64(0), ctypes.byref(info)) == 0x100
    # sort digit width range
    assert lib.gmm_set_sort_digit_bits(3) == 0x100
    assert lib.gmm_set_sort_digit_bits(8) == 0


def test_pybind_surface_has_reference_names():
    import gpu_mm_b200 as g
    m = g.gpu_mm_pybind11
    for name in ("LocalPixelization", "PointingPrePlan", "PointingPlan", "planned_map2tod", "planned_tod2map",
                 "response_map2tod", "response_tod2map", "unplanned_map2tod", "unplanned_tod2map",
                 "reference_map2tod", "reference_tod2map", "expand_dynamic_map", "expand_dynamic_map2",
                 "local_map_to_global", "_get_tsize"):
        assert hasattr(m, name), name
    for name in ("map2tod", "tod2map", "LocalPixelization", "LocalMap", "DynamicMap", "PointingPrePlan",
                 "PointingPlan", "read_xpointing_npzfile"):
        assert hasattr(g, name), name
    assert g.PointingPrePlan.preplan_size == 1024
    for attr in ("nsamp", "nypix_global", "nxpix_global", "periodic_xcoord", "plan_nbytes",
                 "plan_constructor_tmp_nbytes", "overhead", "ncl_per_threadblock", "planner_nblocks",
                 "nmt_per_threadblock", "pointing_nblocks", "plan_nmt", "cub_nbytes", "get_nmt_cumsum"):
        assert hasattr(m.PointingPrePlan, attr), attr


def test_drop_in_import_names():
    """The reference's import names resolve to this build: a caller of the reference writes
    `import gpu_mm` and `from gpu_mm import gpu_mm_pybind11`, unchanged."""
    import importlib
    import gpu_mm_b200
    gm = importlib.import_module("gpu_mm")
    m = importlib.import_module("gpu_mm.gpu_mm_pybind11")
    assert m is gpu_mm_b200.gpu_mm_pybind11 and gm.gpu_mm_pybind11 is m
    from gpu_mm import gpu_mm_pybind11 as m2, map2tod, tod2map, PointingPlan
    assert m2 is m and map2tod is gpu_mm_b200.map2tod and tod2map is gpu_mm_b200.tod2map
    assert PointingPlan is gpu_mm_b200.PointingPlan
    from gpu_mm.gpu_mm import LocalPixelization
    assert LocalPixelization is gpu_mm_b200.LocalPixelization


@pytest.mark.parametrize("ntu", [64, 100, 31, 1])
def test_read_xpointing_npzfile_round_trip(tmp_path, ntu):
    """The reference's .npz pointing format (gpu_mm.py:1305-1329): rows stored as (x, y, alpha) over
    (ndet, nt); read back as (y, x, alpha) with nt padded to a multiple of 32 by repeating each
    detector's last sample."""
    import gpu_mm_b200 as g
    rng = np.random.default_rng(ntu)
    ndet = 3
    stored = rng.standard_normal((3, ndet, ntu)).astype(np.float32)
    path = tmp_path / "xp.npz"
    np.savez(path, xpointing=stored)
    xp = g.read_xpointing_npzfile(str(path))
    ntp = 32 * ((ntu + 31) // 32)
    assert xp.shape == (3, ndet, ntp) and xp.dtype == np.float32
    np.testing.assert_array_equal(xp[0, :, :ntu], stored[1])
    np.testing.assert_array_equal(xp[1, :, :ntu], stored[0])
    np.testing.assert_array_equal(xp[2, :, :ntu], stored[2])
    for r, src in ((0, 1), (1, 0), (2, 2)):
        np.testing.assert_array_equal(xp[r, :, ntu:], np.repeat(stored[src, :, -1:], ntp - ntu, axis=1))
    bad = tmp_path / "bad.npz"
    np.savez(bad, xpointing=stored[:2])
    with pytest.raises(AssertionError):
        g.read_xpointing_npzfile(str(bad))
