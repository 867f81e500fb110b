"""gmm_plan_build_noalloc: plan construction for callers that cannot allocate device memory (a
real-time loop, a host that hands out device memory from its own fixed pool, a foreign runtime
without a device allocator).  It takes its temporary storage from a 32 MiB static device array
instead of a caller-provided buffer.

This file is collected last on purpose; it is self-contained, so it passes alone in a fresh process
as well as after the other tests.  It calls the entry point through the C ABI twice in a row and
compares each plan with the one gmm_plan_build makes from a caller-allocated tmp buffer."""

import ctypes

import numpy as np
import pytest

import oracle
from tests._common import random_raster, rel_stats

pytestmark = pytest.mark.gpu


class Info(ctypes.Structure):
    _fields_ = [("nsamp", ctypes.c_int64), ("nypix_global", ctypes.c_int32), ("nxpix_global", ctypes.c_int32),
                ("periodic_xcoord", ctypes.c_int32), ("sort_digit_bits", ctypes.c_int32),
                ("plan_nbytes", ctypes.c_int64), ("plan_constructor_tmp_nbytes", ctypes.c_int64),
                ("overhead", ctypes.c_double), ("ncl_per_threadblock", ctypes.c_int64),
                ("planner_nblocks", ctypes.c_int64), ("nmt_per_threadblock", ctypes.c_int64),
                ("pointing_nblocks", ctypes.c_int64), ("plan_nmt", ctypes.c_int64), ("sort_nbytes", ctypes.c_int64)]


class Lpix(ctypes.Structure):
    _fields_ = [("nypix_global", ctypes.c_int32), ("nxpix_global", ctypes.c_int32),
                ("periodic_xcoord", ctypes.c_int32), ("nycells", ctypes.c_int32), ("nxcells", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("ystride", ctypes.c_int64), ("polstride", ctypes.c_int64),
                ("npix", ctypes.c_int64), ("cell_offsets", ctypes.c_void_p)]


P = ctypes.c_void_p


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available()
    import gpu_mm_b200
    L = ctypes.CDLL(gpu_mm_b200.library_path())
    L.gmm_last_error.restype = ctypes.c_char_p
    return L


def test_noalloc_plan_matches_allocating_entry_point(lib):
    import torch
    L = lib
    rng = np.random.default_rng(2024)
    ny, nx = 400, 900
    xp = random_raster(rng, 16, 8192, ny, nx, True, speed=0.8)     # 2^17 samples
    nsamp = xp.size // 3
    xg = torch.from_numpy(xp).cuda()
    nmt = torch.zeros(1024, dtype=torch.int32, device="cuda")
    err = torch.zeros(1024, dtype=torch.int32, device="cuda")
    info = Info()
    assert L.gmm_preplan(P(xg.data_ptr()), ctypes.c_int64(nsamp), ny, nx, 1, P(nmt.data_ptr()), P(err.data_ptr()),
                         0, None, ctypes.byref(info)) == 0, L.gmm_last_error()

    # Existing entry point, caller-allocated temporary buffer.
    ref_buf = torch.empty(info.plan_nbytes, dtype=torch.uint8, device="cuda")
    tmp = torch.empty(info.plan_constructor_tmp_nbytes, dtype=torch.uint8, device="cuda")
    assert L.gmm_plan_build(ctypes.byref(info), P(nmt.data_ptr()), P(xg.data_ptr()), P(ref_buf.data_ptr()),
                            ctypes.c_int64(ref_buf.numel()), P(tmp.data_ptr()), ctypes.c_int64(tmp.numel()), 0,
                            None) == 0, L.gmm_last_error()
    torch.cuda.synchronize()

    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    offs = torch.from_numpy(lp_o.cell_offsets).cuda()
    lp = Lpix(ny, nx, 1, lp_o.nycells, lp_o.nxcells, 0, lp_o.ystride, lp_o.polstride, lp_o.npix, offs.data_ptr())
    m = torch.from_numpy(rng.standard_normal(3 * lp_o.npix).astype(np.float32)).cuda()

    def map2tod_with(buf):
        tod = torch.zeros(nsamp, dtype=torch.float32, device="cuda")
        rc = L.gmm_planned_map2tod(P(tod.data_ptr()), P(m.data_ptr()), P(xg.data_ptr()), ctypes.byref(lp),
                                   ctypes.byref(info), P(buf.data_ptr()), 0, 0, None, None)
        assert rc == 0, L.gmm_last_error()
        return tod.cpu().numpy()

    want_tod = map2tod_with(ref_buf)
    want_buf = ref_buf.cpu().numpy()
    for _ in range(2):   # two calls in a row share (and reuse) the static scratch
        buf = torch.full((info.plan_nbytes,), 0x5A, dtype=torch.uint8, device="cuda")
        rc = L.gmm_plan_build_noalloc(ctypes.byref(info), P(nmt.data_ptr()), P(xg.data_ptr()), P(buf.data_ptr()),
                                      ctypes.c_int64(buf.numel()), 0, None)
        assert rc == 0, L.gmm_last_error()
        torch.cuda.synchronize()
        # The plan is integer data: identical bit for bit, including the owner list and cell bitmap.
        np.testing.assert_array_equal(buf.cpu().numpy()[:8 * info.plan_nmt], want_buf[:8 * info.plan_nmt])
        got = map2tod_with(buf)
        rl1, mx = rel_stats(got, want_tod)
        assert rl1 < 1e-6 and mx < 1e-5


def test_noalloc_rejects_oversized_plans(lib):
    L = lib
    info = Info()
    # 2^28 samples: far more temporary storage than the 32 MiB static scratch.
    assert L.gmm_preplan_info_init(ctypes.c_int64(1 << 28), 8192, 32768, 1, ctypes.c_int64(11 << 20),
                                   ctypes.byref(info)) == 0
    assert info.plan_constructor_tmp_nbytes > (32 << 20)
    rc = L.gmm_plan_build_noalloc(ctypes.byref(info), P(256), P(256), P(256), ctypes.c_int64(info.plan_nbytes), 0,
                                  None)
    assert rc == 0x400
    assert b"static scratch" in L.gmm_last_error()
