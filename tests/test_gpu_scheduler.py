"""Every cache line is visited exactly once by every planned operator kernel, whatever the shape of the
owner list: the analogue of the reference's plan-iterator test (test_plan_iterator.cu:120-167,
tests.py:16-25), which checks that a random plan visits each mt word once.

The pointing is integer-valued (every sample sits exactly on a pixel, so its bilinear weights are
(1, 0, 0, 0)) and alpha = 0 (cos 2a = 1, sin 2a = 0).  Then
  * map2tod of the map (T, Q, U) = (1, 0, 0) with accum adds exactly 1.0 to every sample, and
  * tod2map of an all-ones TOD puts the exact hit count of each pixel into T and Q,
so a line visited twice or never shows up as an exact integer mismatch.

Lines are spread over the cells with a heavy-tailed number of lines per cell (many cells with one
line, a few with hundreds), so cell runs start and end anywhere relative to the operators' CTA and
warp slices; line shapes mix constant x, runs of one to four samples per column, both directions,
and lines that cross a cell boundary.  The tile kernel is also run with the precision modes and a
small max_run_lines, which splits cell runs further, and so is the mode that reduces the partials of
high-hit cells in float64.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GMM_TOD2MAP_BANDS = 0
GMM_TOD2MAP_TILES = 1


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


def integer_lines(seed, nlines, ny, nx):
    """(3, nlines*32) float32 integer pointing, one random cell per line (Zipf-like line counts)."""
    rng = np.random.default_rng(seed)
    nyc, nxc = ny // 64, nx // 64
    ncells = nyc * nxc
    weights = 1.0 / np.arange(1, ncells + 1) ** 1.3
    cells = rng.permutation(ncells)[rng.choice(ncells, size=nlines, p=weights / weights.sum())]
    i = np.arange(32)
    xp = np.zeros((3, nlines, 32))
    for l, c in enumerate(cells):
        cy, cx = divmod(int(c), nxc)
        kind = rng.integers(0, 7)
        y0 = 64 * cy + rng.integers(0, 63)
        x0 = 64 * cx + rng.integers(0, 64)
        if kind == 0:
            x = np.full(32, x0)                      # one pixel for the whole line
        elif kind in (1, 2, 3, 4):
            x = x0 + i // kind                       # runs of 1..4 samples per column
        elif kind == 5:
            x = x0 + 31 - i // 2                     # decreasing
        else:
            x = x0 + (i * 2) // 3 + (i >= 16) * 3    # a jump of 3 columns in the middle
        y = np.full(32, y0) + ((i >= 20) & (rng.random() < 0.3))   # some lines step down a row
        xp[0, l] = np.minimum(y, ny - 2)
        xp[1, l] = np.minimum(x, nx - 3)
    return xp.reshape(3, -1).astype(np.float32)


def expected_counts(xp, ny, nx):
    """Hits per pixel as (ny, nx); make_rectangle's local map is the global map in row-major order."""
    y = xp[0].astype(np.int64)
    x = xp[1].astype(np.int64)
    cnt = np.zeros(ny * nx, np.float64)
    np.add.at(cnt, y * nx + x, 1.0)
    return cnt.reshape(ny, nx)


@pytest.mark.parametrize("seed,nlines", [(0, 37), (1, 1000), (2, 4097), (3, 30000)])
def test_each_line_exactly_once(g, kernel_knob, seed, nlines):
    import torch
    ny, nx = 512, 1024
    xp = integer_lines(seed, nlines, ny, nx)
    want = expected_counts(xp, ny, nx)
    xg = torch.from_numpy(xp).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=False)
    plan = g.PointingPlan(pp, xg)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    rng = np.random.default_rng(100 + seed)

    # map2tod with accum: +1 per visit, for both map2tod kernels (16-byte aligned and not).
    m = np.zeros((3, ny, nx), np.float32)
    m[0] = 1.0
    lmap = g.LocalMap(lp, torch.from_numpy(m.ravel()).cuda())
    t0 = rng.integers(-1000, 1000, size=xp.shape[1]).astype(np.float32)
    tod = torch.from_numpy(t0).cuda()
    g.map2tod(tod, lmap, xg, plan, accum=True)
    np.testing.assert_array_equal(tod.cpu().numpy(), t0 + 1.0)
    buf = torch.zeros(xp.shape[1] + 1, device="cuda")
    tod_odd = buf[1:]                                   # not 16-byte aligned: the scalar kernel
    tod_odd.copy_(torch.from_numpy(t0))
    g.map2tod(tod_odd, lmap, xg, plan, accum=True)
    np.testing.assert_array_equal(tod_odd.cpu().numpy(), t0 + 1.0)

    ones = torch.ones(xp.shape[1], device="cuda")
    for which in (GMM_TOD2MAP_BANDS, GMM_TOD2MAP_TILES):
        kernel_knob(which)
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map(out, ones, xg, plan)
        got = out.arr.cpu().numpy().reshape(3, ny, nx)
        np.testing.assert_array_equal(got[0], want, err_msg=f"T, kernel {which}")
        np.testing.assert_array_equal(got[1], want, err_msg=f"Q, kernel {which}")
        assert not np.any(got[2]), f"U, kernel {which}"

    # Precision modes with short runs: cell runs are split every max_run_lines lines.
    for mrl in (1, 3, 64):
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        comp = torch.zeros(3 * lp.npix, device="cuda")
        g.tod2map_compensated(out, comp, ones, xg, plan, max_run_lines=mrl)
        g.fold_compensation(out, comp)
        got = out.arr.cpu().numpy().reshape(3, ny, nx)
        np.testing.assert_array_equal(got[0], want, err_msg=f"compensated, max_run_lines {mrl}")
        m64 = torch.zeros(3 * lp.npix, dtype=torch.float64, device="cuda")
        g.tod2map_f64(m64, lp, ones, xg, plan, max_run_lines=mrl)
        got = m64.cpu().numpy().reshape(3, ny, nx)
        np.testing.assert_array_equal(got[0], want, err_msg=f"float64 map, max_run_lines {mrl}")

    # float64 only in the cells touched by at least the median number of lines (the rest take float
    # atomics).
    lines = g.HotCells(lp, [plan], 0).lines()
    hot = g.HotCells(lp, [plan], max(1, int(np.median(lines[lines > 0]))))
    assert 0 < hot.nhot < lp.nycells * lp.nxcells
    for mrl in (0, 1, 3):
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map_hot_f64(out, hot, ones, xg, plan, max_run_lines=mrl)
        hot.fold(out)
        got = out.arr.cpu().numpy().reshape(3, ny, nx)
        np.testing.assert_array_equal(got[0], want, err_msg=f"hot cells, max_run_lines {mrl}")
        np.testing.assert_array_equal(got[1], want, err_msg=f"hot cells Q, max_run_lines {mrl}")
