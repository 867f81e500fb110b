"""GPU tests of the double-precision unplanned operators (gmm_unplanned_map2tod_f64 /
gmm_unplanned_tod2map_f64, the reference's launch_unplanned_*<double>), called through the C ABI
and compared with the oracle's float64 operators (reference_map2tod<double> semantics).  Double
accumulation leaves only reordering differences, so the tolerance is 1e-12."""

import ctypes

import numpy as np
import pytest

import oracle
from tests._common import random_raster, rel_stats

pytestmark = pytest.mark.gpu

TOL = 1e-12
P = ctypes.c_void_p


class Lpix(ctypes.Structure):
    _fields_ = [("nypix_global", ctypes.c_int32), ("nxpix_global", ctypes.c_int32),
                ("periodic_xcoord", ctypes.c_int32), ("nycells", ctypes.c_int32), ("nxcells", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("ystride", ctypes.c_int64), ("polstride", ctypes.c_int64),
                ("npix", ctypes.c_int64), ("cell_offsets", ctypes.c_void_p)]


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available()
    import gpu_mm_b200
    L = ctypes.CDLL(gpu_mm_b200.library_path())
    L.gmm_last_error.restype = ctypes.c_char_p
    return L


def device_lpix(lp_o, periodic, keep):
    import torch
    offs = torch.from_numpy(np.ascontiguousarray(lp_o.cell_offsets)).cuda()
    return Lpix(lp_o.nypix_global, lp_o.nxpix_global, int(periodic), lp_o.nycells, lp_o.nxcells, 0, lp_o.ystride,
                lp_o.polstride, lp_o.npix, offs.data_ptr()), offs


@pytest.mark.parametrize("periodic,accum", [(True, False), (False, True)])
def test_unplanned_f64_matches_oracle(lib, periodic, accum):
    import torch
    L = lib
    rng = np.random.default_rng(64 + int(periodic))
    ny, nx = 256, 512
    xp = random_raster(rng, 6, 4000, ny, nx, periodic).astype(np.float64)
    nsamp = xp.size // 3
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    lp, offs = device_lpix(lp_o, periodic, True)
    m = rng.standard_normal(3 * lp_o.npix)
    tod0 = rng.standard_normal(xp.shape[1:])
    errflags = torch.zeros(4, dtype=torch.int32, device="cuda")
    xg, mg = torch.from_numpy(xp).cuda(), torch.from_numpy(m).cuda()

    # map2tod
    tod = torch.from_numpy(tod0.copy()).cuda()
    rc = L.gmm_unplanned_map2tod_f64(P(tod.data_ptr()), P(mg.data_ptr()), P(xg.data_ptr()), ctypes.c_int64(nsamp),
                                     ctypes.byref(lp), P(errflags.data_ptr()), ctypes.c_int64(4), 0, int(accum), 1,
                                     None)
    assert rc == 0, L.gmm_last_error()
    want = tod0.copy()
    oracle.map2tod(want, m, xp, lp_o, accum=accum)
    rl1, mx = rel_stats(tod.cpu().numpy(), want)
    assert rl1 < TOL and mx < TOL, (rl1, mx)

    # tod2map (accumulates into the map)
    out = torch.from_numpy(m.copy()).cuda()
    rc = L.gmm_unplanned_tod2map_f64(P(out.data_ptr()), P(torch.from_numpy(tod0).cuda().data_ptr()),
                                     P(xg.data_ptr()), ctypes.c_int64(nsamp), ctypes.byref(lp),
                                     P(errflags.data_ptr()), ctypes.c_int64(4), 0, 1, None)
    assert rc == 0, L.gmm_last_error()
    want_m = m.copy()
    oracle.tod2map(want_m, tod0, xp, lp_o)
    rl1, mx = rel_stats(out.cpu().numpy() - m, want_m - m)
    assert rl1 < TOL and mx < TOL, (rl1, mx)


def test_unplanned_f64_errors(lib):
    import torch
    L = lib
    rng = np.random.default_rng(3)
    ny, nx = 128, 256
    xp = random_raster(rng, 2, 1024, ny, nx, False).astype(np.float64)
    nsamp = xp.size // 3
    xp[0, 1, 17] = ny + 3.0                        # y outside the map
    lp_o = oracle.Lpix.rectangle(ny, nx, False)
    lp, offs = device_lpix(lp_o, False, True)
    errflags = torch.zeros(1, dtype=torch.int32, device="cuda")
    tod = torch.zeros(xp.shape[1:], dtype=torch.float64, device="cuda")
    m = torch.zeros(3 * lp_o.npix, dtype=torch.float64, device="cuda")
    rc = L.gmm_unplanned_map2tod_f64(P(tod.data_ptr()), P(m.data_ptr()), P(torch.from_numpy(xp).cuda().data_ptr()),
                                     ctypes.c_int64(nsamp), ctypes.byref(lp), P(errflags.data_ptr()),
                                     ctypes.c_int64(1), 0, 0, 1, None)
    assert rc == 1 and b"y-value" in L.gmm_last_error()
    # Bad arguments are refused before any device work.
    rc = L.gmm_unplanned_tod2map_f64(None, P(tod.data_ptr()), P(tod.data_ptr()), ctypes.c_int64(nsamp),
                                     ctypes.byref(lp), P(errflags.data_ptr()), ctypes.c_int64(1), 0, 1, None)
    assert rc != 0
