"""GPU tests of the tod2map precision variants (float atomics, compensated float flush, float64 map,
float64 only in the high-hit cells) against the FP64 oracle (reference_tod2map<double> semantics on
the float32 inputs widened).

Errors are stated per map: max relative error = max|a-b| / max|b| and rms relative error =
sqrt(sum (a-b)^2 / sum b^2), over all three planes.
"""

import numpy as np
import pytest

import oracle
from tests._common import random_raster, rel_stats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200
    return gpu_mm_b200


def err_vs(a, ref):
    a = np.asarray(a, np.float64)
    d = a - ref
    return float(np.abs(d).max() / np.abs(ref).max()), float(np.sqrt((d * d).sum() / (ref * ref).sum()))


def high_hit_case(seed, ndet_side=4, nt=65536, box=64, ny=256, nx=256):
    """A narrow raster confined to a box x box patch (x bounces at 0.7 px/sample, y at an
    incommensurate 0.0123 px/sample) with a large DC offset in the TOD: tod = 1e3 + N(0,1).
    About nsamp*4/box^2 hits per pixel."""
    import torch
    from gpu_mm_b200 import synthetic
    xp = synthetic.raster_xpointing(ndet_side, ndet_side, nt, 2.0, 0.7, nx, 96.0, 0.0, xlo=96.0,
                                    xspan=box - 1.0 - 2.0 * ndet_side, yspan=box - 1.0 - 2.0 * ndet_side,
                                    yspeed=0.0123, wrap_x=False, device="cpu").numpy()
    rng = np.random.default_rng(seed)
    tod = (1e3 + rng.standard_normal(xp.shape[1:])).astype(np.float32)
    return xp, tod, ny, nx


def run_modes(g, xp, tod, ny, nx, max_run_lines):
    import torch
    xg = torch.from_numpy(xp).cuda()
    tg = torch.from_numpy(tod).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=False)
    plan = g.PointingPlan(pp, xg)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    out = {}
    m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    g.tod2map(m, tg, xg, plan)
    out["fp32"] = m.arr.cpu().numpy()
    m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    comp = torch.zeros(3 * lp.npix, device="cuda")
    g.tod2map_compensated(m, comp, tg, xg, plan, max_run_lines=max_run_lines)
    g.fold_compensation(m, comp)
    assert float(comp.abs().max()) == 0.0
    out["compensated"] = m.arr.cpu().numpy()
    m64 = torch.zeros(3 * lp.npix, dtype=torch.float64, device="cuda")
    g.tod2map_f64(m64, lp, tg, xg, plan, max_run_lines=max_run_lines)
    out["fp64map"] = m64.cpu().numpy()
    return out


def test_precision_modes_high_hit(g):
    xp, tod, ny, nx = high_hit_case(31)
    lp_o = oracle.Lpix.rectangle(ny, nx, False)
    want = np.zeros(3 * lp_o.npix, np.float64)
    assert oracle.tod2map_f64w_mt(want, tod, xp, lp_o, 8) == 0
    out = run_modes(g, xp, tod, ny, nx, max_run_lines=64)
    errs = {k: err_vs(v, want) for k, v in out.items()}
    # Compensated and float64 reductions leave only the float tile partials (<= 64 lines each).
    for k in ("compensated", "fp64map"):
        assert errs[k][0] < 1e-5 and errs[k][1] < 1e-6, (k, errs)
    assert errs["fp64map"][1] <= errs["fp32"][1], errs
    assert errs["compensated"][1] <= errs["fp32"][1], errs


def test_precision_modes_match_float_path(g):
    """On an ordinary scan (periodic, fast enough that some footprints leave the tile and take the
    global path) every mode agrees with the float oracle at the float operators' tolerance."""
    import torch
    rng = np.random.default_rng(4242)
    ny, nx = 256, 512
    xp = random_raster(rng, 12, 2048, ny, nx, True, speed=1.6)
    tod = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    want = np.zeros(3 * lp_o.npix, np.float32)
    oracle.tod2map(want, tod, xp, lp_o)
    xg = torch.from_numpy(xp).cuda()
    tg = torch.from_numpy(tod).cuda()
    pp = g.PointingPrePlan(xg, ny, nx)
    plan = g.PointingPlan(pp, xg)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    for max_run_lines in (0, 7):
        m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        comp = torch.zeros(3 * lp.npix, device="cuda")
        g.tod2map_compensated(m, comp, tg, xg, plan, max_run_lines=max_run_lines)
        g.fold_compensation(m, comp)
        rl1, mx = rel_stats(m.arr.cpu().numpy(), want)
        assert rl1 < 1e-6 and mx < 1e-5, ("compensated", max_run_lines, rl1, mx)
        m64 = torch.zeros(3 * lp.npix, dtype=torch.float64, device="cuda")
        g.tod2map_f64(m64, lp, tg, xg, plan, max_run_lines=max_run_lines)
        rl1, mx = rel_stats(m64.cpu().numpy().astype(np.float32), want)
        assert rl1 < 1e-6 and mx < 1e-5, ("fp64map", max_run_lines, rl1, mx)


def test_precision_argument_checks(g):
    import torch
    rng = np.random.default_rng(1)
    xp = random_raster(rng, 2, 256, 128, 128, True)
    xg = torch.from_numpy(xp).cuda()
    pp = g.PointingPrePlan(xg, 128, 128)
    plan = g.PointingPlan(pp, xg)
    lp = g.LocalPixelization.make_rectangle(128, 128, True)
    m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    tg = torch.zeros(xp.shape[1:], device="cuda")
    with pytest.raises(RuntimeError):
        g.tod2map_compensated(m, torch.zeros(5, device="cuda"), tg, xg, plan)
    with pytest.raises(RuntimeError):
        g.tod2map_compensated(m, torch.zeros(3 * lp.npix, device="cuda"), tg, xg, plan, max_run_lines=-1)
    with pytest.raises(RuntimeError):
        g.tod2map_f64(torch.zeros(3 * lp.npix, dtype=torch.float32, device="cuda"), lp, tg, xg, plan)


def test_precision_modes_full_size_high_hit(g):
    """The high-hit precision workload at its full size: 64 detectors x 2^22 samples (2^28) confined to
    the 512x512 box [256, 768)^2 of a 3x1024x1024 map (~1000 hits/pixel), tod = 1e3 + N(0,1), against
    the FP64 oracle over the whole TOD.  Bars: a 1e-5 max relative error for the float
    path (both tod2map kernels); 1e-6 max and 2e-7 rms for the compensated and float64-map modes on
    both kernels, with float partials of at most 32 lines (max_run_lines)."""
    import ctypes
    import os
    import torch
    from gpu_mm_b200 import synthetic
    ny = nx = 1024
    xg = synthetic.config3_xpointing(device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(3)
    tg = 1e3 + torch.randn(xg.shape[1:], generator=gen, device="cuda")
    lp_o = oracle.Lpix.rectangle(ny, nx, False)
    want = np.zeros(3 * lp_o.npix, np.float64)
    assert oracle.tod2map_f64w_mt(want, tg.cpu().numpy(), xg.cpu().numpy(), lp_o, os.cpu_count() or 1) == 0
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=False)
    plan = g.PointingPlan(pp, xg)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    lib = ctypes.CDLL(g.library_path())
    old = lib.gmm_get_planned_tod2map_kernel()
    errs = {}
    try:
        for which in (0, 1):
            lib.gmm_set_planned_tod2map_kernel(which)
            m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
            g.tod2map(m, tg, xg, plan)
            errs[f"fp32-{which}"] = err_vs(m.arr.cpu().numpy(), want)
        for which in (0, 1):
            lib.gmm_set_planned_tod2map_kernel(which)
            m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
            comp = torch.zeros(3 * lp.npix, device="cuda")
            g.tod2map_compensated(m, comp, tg, xg, plan, max_run_lines=32)
            g.fold_compensation(m, comp)
            errs[f"compensated-{which}"] = err_vs(m.arr.cpu().numpy(), want)
            m64 = torch.zeros(3 * lp.npix, dtype=torch.float64, device="cuda")
            g.tod2map_f64(m64, lp, tg, xg, plan, max_run_lines=32)
            errs[f"fp64map-{which}"] = err_vs(m64.cpu().numpy(), want)
    finally:
        lib.gmm_set_planned_tod2map_kernel(old)
    for k in ("fp32-0", "fp32-1"):
        assert errs[k][0] < 1e-5, (k, errs)
    for k in ("compensated-0", "compensated-1", "fp64map-0", "fp64map-1"):
        assert errs[k][0] < 1e-6 and errs[k][1] < 2e-7, (k, errs)


def hot_lines_and_slots(plans, present, min_lines):
    """numpy restatement of HotCells: per cell of the grid the number of plan mt words (cache lines
    touching the cell); slots in cell order over the present cells with at least min_lines."""
    nyc, nxc = present.shape
    lines = np.zeros(nyc * nxc, np.int64)
    for p in plans:
        mt = p.get_plan_mt().astype(np.uint64)
        ixc = (mt & np.uint64(1023)).astype(np.int64)
        iyc = ((mt >> np.uint64(10)) & np.uint64(1023)).astype(np.int64)
        ok = (iyc < nyc) & (ixc < nxc)
        lines += np.bincount(iyc[ok] * nxc + ixc[ok], minlength=nyc * nxc)
    hot = (lines >= min_lines) & present.ravel()
    slot = np.where(hot, np.cumsum(hot) - 1, -1)
    return lines.reshape(nyc, nxc), slot.reshape(nyc, nxc)


def test_hot_cells_mixed_depth(g):
    """float64 only in the high-hit cells: a deep TOD (~1000 hits/pixel in a 64x64-cell-aligned box)
    and a shallow TOD over the whole map go into one float map.  With a threshold between the two
    depths the box's cells are hot: their error against the FP64 oracle is that of the float64 map
    mode (max rel < 1e-6), the other cells keep float atomics, and the whole map is within the float
    path's bar.  min_lines = 0 makes every present cell hot; a threshold above every count none."""
    import torch
    ny, nx = 256, 256
    xd, td, _, _ = high_hit_case(77)                 # the deep box is [96, 160)^2 (cells 1..2)
    rng = np.random.default_rng(78)
    xw = random_raster(rng, 8, 8192, ny, nx, False, speed=0.7, ydrift=0.02)
    tw = (1e3 + rng.standard_normal(xw.shape[1:])).astype(np.float32)
    lp_o = oracle.Lpix.rectangle(ny, nx, False)
    want = np.zeros(3 * lp_o.npix, np.float64)
    for xp, tod in ((xd, td), (xw, tw)):
        assert oracle.tod2map_f64w_mt(want, tod, xp, lp_o, 8) == 0
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    todos = []
    for xp, tod in ((xd, td), (xw, tw)):
        xg = torch.from_numpy(xp).cuda()
        pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=False)
        todos.append((xg, torch.from_numpy(tod).cuda(), g.PointingPlan(pp, xg)))
    plans = [p for _, _, p in todos]
    present = np.ones((lp.nycells, lp.nxcells), bool)
    lines_ref, _ = hot_lines_and_slots(plans, present, 0)
    deep = lines_ref.max()
    threshold = int(deep // 4)
    results = {}
    for min_lines in (0, threshold, int(deep) + 1):
        hot = g.HotCells(lp, plans, min_lines)
        lines, slot = hot_lines_and_slots(plans, present, min_lines)
        np.testing.assert_array_equal(hot.lines(), lines)
        np.testing.assert_array_equal(hot.slots(), slot)
        assert hot.nhot == int((slot >= 0).sum())
        m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        for xg, tg, plan in todos:
            g.tod2map_hot_f64(m, hot, tg, xg, plan, max_run_lines=32)
        hot.fold(m)
        results[min_lines] = (m.arr.cpu().numpy(), slot)
    assert results[0][1].min() == 0 and (results[int(deep) + 1][1] < 0).all()
    got, slot = results[threshold]
    hot_mask = np.broadcast_to((slot >= 0)[:, None, :, None], (lp.nycells, 64, lp.nxcells, 64)).reshape(ny, nx)
    assert 0 < hot_mask.mean() < 0.5
    w3, g3 = want.reshape(3, ny, nx), got.reshape(3, ny, nx)
    scale = np.abs(want).max()
    hot_err = np.abs(g3 - w3)[:, hot_mask].max() / scale
    cold_err = np.abs(g3 - w3)[:, ~hot_mask].max() / scale
    assert hot_err < 1e-6, (hot_err, cold_err)
    assert err_vs(got, want)[0] < 1e-5
    # All hot: float64 reductions everywhere, one rounding at the fold.
    e_all = err_vs(results[0][0], want)
    assert e_all[0] < 1e-6 and e_all[1] < 2e-7, e_all
    # None hot: the float path.
    e_none = err_vs(results[int(deep) + 1][0], want)
    assert e_none[0] < 1e-5, e_none
    # The float path's error in the box is what the hot cells remove.
    assert hot_err <= np.abs(results[int(deep) + 1][0].reshape(3, ny, nx) - w3)[:, hot_mask].max() / scale


def test_hot_cells_absent_cells_and_checks(g):
    """Absent cells are never hot and drop their samples with partial_pixelization (and raise without
    it); tod2map_hot_f64 needs 16-byte aligned arrays and the HotCells of the map's pixelization."""
    import torch
    rng = np.random.default_rng(9)
    ny, nx = 256, 512
    xp = random_raster(rng, 8, 4096, ny, nx, True)
    tod = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    offs = np.full((4, 8), -1, np.int64)
    k = 0
    for iy in range(4):
        for ix in range(8):
            if (iy + 2 * ix) % 5 != 2:
                offs[iy, ix] = 3 * 4096 * k
                k += 1
    lp = g.LocalPixelization(ny, nx, offs, 64, 4096, True)
    lp_o = oracle.Lpix(ny, nx, offs, 64, 4096, True)
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, tod, xp, lp_o, True)
    xg = torch.from_numpy(xp).cuda()
    tg = torch.from_numpy(tod).cuda()
    pp = g.PointingPrePlan(xg, ny, nx)
    plan = g.PointingPlan(pp, xg)
    hot = g.HotCells(lp, [plan], 1)
    _, slot = hot_lines_and_slots([plan], offs >= 0, 1)
    np.testing.assert_array_equal(hot.slots(), slot)
    assert (hot.slots()[offs < 0] == -1).all()
    m = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    g.tod2map_hot_f64(m, hot, tg, xg, plan, partial_pixelization=True, max_run_lines=5)
    hot.fold(m)
    rl1, mx = rel_stats(m.arr.cpu().numpy(), want)
    assert rl1 < 1e-6 and mx < 1e-5, (rl1, mx)
    with pytest.raises(RuntimeError, match="not in LocalPixelization"):
        g.tod2map_hot_f64(m, hot, tg, xg, plan, partial_pixelization=False)
    buf = torch.zeros(tg.numel() + 1, device="cuda")
    with pytest.raises(RuntimeError, match="16-byte aligned"):
        g.tod2map_hot_f64(m, hot, buf[1:].reshape(tg.shape), xg, plan, partial_pixelization=True)
    lp2 = g.LocalPixelization.make_rectangle(ny, nx, True)
    with pytest.raises(RuntimeError):
        g.tod2map_hot_f64(g.LocalMap(lp2, torch.zeros(3 * lp2.npix, device="cuda")), hot, tg, xg, plan)
