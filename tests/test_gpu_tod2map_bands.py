"""Planned tod2map on both of its kernels -- row bands (the default for single-TOD plans) and
shared-memory tiles -- and unplanned tod2map against the oracle, on scans chosen to reach every
branch of the band path and of the unplanned line path:
scan speeds giving one to four samples per pixel column and more (which the band path leaves to
its per-sample route), both scan directions, turnarounds, x wraparound, lines that cross a pixel
row (the band path's two-row pass, y increasing and decreasing), absent cells, and the
per-detector response.

Tolerances are those of the other parity tests: rel-L1 < 1e-6 (the reference's metric,
tests.py:220-224) and max|a-b| / max|b| < 1e-5.
"""

import ctypes

import numpy as np
import pytest

import oracle
from tests._common import rel_stats

pytestmark = pytest.mark.gpu

RL1_TOL = 1e-6
MAX_TOL = 1e-5
KERNELS = (0, 1)   # GMM_TOD2MAP_BANDS, GMM_TOD2MAP_TILES


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200
    return gpu_mm_b200


@pytest.fixture
def kernel_knob(g):
    lib = ctypes.CDLL(g.library_path())
    old = lib.gmm_get_planned_tod2map_kernel()

    def set_kernel(which):
        assert lib.gmm_set_planned_tod2map_kernel(which) == 0
    yield set_kernel
    lib.gmm_set_planned_tod2map_kernel(old)


def bounce_scan(rng, ndet, nt, ny, nx, periodic, speed, ydrift, spacing=2.0):
    """Detectors on a line in x (spacing px); x bounces over the map at 'speed' px/sample, y drifts.
    With periodic x the scan is shifted so that some lines cross x = nx."""
    t = np.arange(nt, dtype=np.float64)
    L = nx - 3.0 - spacing * ndet
    xp = np.zeros((3, ndet, nt))
    y0 = rng.uniform(1.0, ny - 3.0 - abs(ydrift) * nt - 0.37 * ndet) + max(0.0, -ydrift) * nt
    ph = rng.uniform(0, 2 * L)
    for d in range(ndet):
        x = np.abs(np.remainder(speed * t + ph, 2 * L) - L) + spacing * d
        if periodic:
            x = np.remainder(x + 0.6 * nx, nx)
        xp[0, d] = y0 + ydrift * t + 0.37 * d
        xp[1, d] = x
        xp[2, d] = 2 * np.pi * np.remainder(t / 777.0 + d / ndet, 1.0)
    return xp.astype(np.float32)


CASES = [
    # (speed, ydrift, periodic, ny, nx)
    (0.7, 2e-4, True, 256, 1024),
    (0.7, 2e-4, False, 256, 1024),
    (0.26, 1e-4, True, 200, 512),      # four samples per column
    (0.34, 0.0, False, 200, 512),      # three
    (0.5, 3e-3, True, 300, 700),       # lines cross pixel rows often
    (0.99, 0.0, True, 128, 600),
    (1.6, 0.0, True, 128, 600),        # faster than a pixel per sample: per-sample route
    (0.18, 0.0, True, 128, 256),       # five or more per column: per-sample route
    (0.7, 0.02, True, 400, 1024),      # y drifts 0.64 px per line: most lines cross a pixel row
    (0.6, -0.015, False, 400, 700),    # the same, y decreasing
]


@pytest.mark.parametrize("case", CASES)
def test_bands_vs_tiles_vs_oracle(g, kernel_knob, case):
    import torch
    speed, ydrift, periodic, ny, nx = case
    rng = np.random.default_rng(int(1000 * speed) + ny)
    xp = bounce_scan(rng, 12, 8192, ny, nx, periodic, speed, ydrift)
    xg = torch.from_numpy(xp).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    if abs(ydrift) >= 0.01:
        bw = plan._get_band_words()
        assert np.mean((bw >> np.uint64(48)) & np.uint64(1)) > 0.3   # lines on the two-row band path
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    t = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    m0 = rng.standard_normal(3 * lp.npix).astype(np.float32)
    want = m0.copy()
    oracle.tod2map(want, t, xp, lp_o)
    tg = torch.from_numpy(t).cuda()
    for which in KERNELS:
        kernel_knob(which)
        out = g.LocalMap(lp, torch.from_numpy(m0).cuda())
        g.tod2map(out, tg, xg, plan)
        rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (which, rl1, mx)
    # The unplanned operator's line path takes the same scans (runs of one to four samples per column).
    out = g.LocalMap(lp, torch.from_numpy(m0).cuda())
    g.tod2map(out, tg, xg, None)
    rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, ("unplanned", rl1, mx)


def test_bands_absent_cells_and_response(g, kernel_knob):
    """Cells missing from the local map are skipped (with partial_pixelization) or raise, and the
    per-detector response weights T and P (tod2map_response.cu) on both kernels."""
    import torch
    rng = np.random.default_rng(5)
    ny, nx, periodic = 256, 512, True
    xp = bounce_scan(rng, 8, 4096, ny, nx, periodic, 0.6, 5e-4)
    xg = torch.from_numpy(xp).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    nyc, nxc = 4, 8
    offs = np.full((nyc, nxc), -1, np.int64)
    k = 0
    for iy in range(nyc):
        for ix in range(nxc):
            if (iy * 5 + ix * 3) % 4 != 1:
                offs[iy, ix] = 3 * 4096 * k
                k += 1
    lp = g.LocalPixelization(ny, nx, offs, 64, 4096, periodic)
    lp_o = oracle.Lpix(ny, nx, offs, 64, 4096, periodic)
    t = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    tg = torch.from_numpy(t).cuda()
    want = np.zeros(3 * lp.npix, np.float32)
    err = oracle.tod2map(want, t, xp, lp_o, False)     # same values as partial=True, plus the error bit
    assert err & oracle.ERR_NOT_IN_PIXELIZATION
    resp = rng.uniform(0.5, 1.5, size=(2, 8)).astype(np.float32)
    want_r = np.zeros(3 * lp.npix, np.float32)
    oracle.response_tod2map(want_r, t, xp, resp, lp_o, True)
    for which in KERNELS:
        kernel_knob(which)
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map(out, tg, xg, plan, partial_pixelization=True)
        rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (which, rl1, mx)
        with pytest.raises(RuntimeError, match="not in LocalPixelization"):
            g.tod2map(out, tg, xg, plan, partial_pixelization=False)
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map(out, tg, xg, plan, partial_pixelization=True, response=torch.from_numpy(resp).cuda())
        rl1, mx = rel_stats(out.arr.cpu().numpy(), want_r)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("response", which, rl1, mx)


def test_absent_cell_in_every_cell_row(g, kernel_knob):
    """The not-in-pixelization check covers the plan's whole cell bitmap on both tod2map kernels and
    in map2tod, whatever their block sizes: scans through cell rows 0..15 of a 1024-row map, one absent
    cell in each of rows 5, 12 and 15."""
    import torch
    rng = np.random.default_rng(12)
    ny, nx, periodic = 1024, 512, True
    for row in (5, 12, 15):
        xp = bounce_scan(rng, 8, 4096, ny, nx, periodic, 0.6, 0.0)
        xp[0] += 64.0 * row + 20.0 - xp[0].min()          # into cell row 'row'
        xg = torch.from_numpy(xp).cuda()
        pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
        plan = g.PointingPlan(pp, xg)
        cx = int(np.floor(xp[1, 0, 0] / 64.0))
        o = np.full((16, 8), -1, np.int64)
        k = 0
        for iy in range(16):
            for ix in range(8):
                if (iy, ix) != (row, cx):
                    o[iy, ix] = 3 * 4096 * k
                    k += 1
        lp = g.LocalPixelization(ny, nx, o, 64, 4096, periodic)
        tg = torch.from_numpy(rng.standard_normal(xp.shape[1:]).astype(np.float32)).cuda()
        for which in KERNELS:
            kernel_knob(which)
            out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
            with pytest.raises(RuntimeError, match="not in LocalPixelization"):
                g.tod2map(out, tg, xg, plan, partial_pixelization=False)
        with pytest.raises(RuntimeError, match="not in LocalPixelization"):
            g.map2tod(torch.zeros(xp.shape[1:], device="cuda"), g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda")),
                      xg, plan, partial_pixelization=False)



def test_bands_response_on_row_crossing_lines(g, kernel_knob):
    """The per-detector response on the band path's two-row pass (y drifting 0.64 px per line), both
    kernels, and the precision modes on the same lines, against the oracle."""
    import torch
    rng = np.random.default_rng(17)
    ny, nx, periodic = 400, 1024, True
    xp = bounce_scan(rng, 12, 4096, ny, nx, periodic, 0.7, 0.02)
    xg = torch.from_numpy(xp).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    bw = plan._get_band_words()
    assert np.mean((bw >> np.uint64(48)) & np.uint64(1)) > 0.3
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    t = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    tg = torch.from_numpy(t).cuda()
    resp = rng.uniform(0.5, 1.5, size=(2, 12)).astype(np.float32)
    want_r = np.zeros(3 * lp.npix, np.float32)
    oracle.response_tod2map(want_r, t, xp, resp, lp_o, False)
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, t, xp, lp_o)
    for which in KERNELS:
        kernel_knob(which)
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map(out, tg, xg, plan, response=torch.from_numpy(resp).cuda())
        rl1, mx = rel_stats(out.arr.cpu().numpy(), want_r)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("response", which, rl1, mx)
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        comp = torch.zeros(3 * lp.npix, device="cuda")
        g.tod2map_compensated(out, comp, tg, xg, plan, max_run_lines=5)
        g.fold_compensation(out, comp)
        rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("compensated", which, rl1, mx)
        m64 = torch.zeros(3 * lp.npix, dtype=torch.float64, device="cuda")
        g.tod2map_f64(m64, lp, tg, xg, plan, max_run_lines=5)
        rl1, mx = rel_stats(m64.cpu().numpy().astype(np.float32), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("float64", which, rl1, mx)
