"""GPU tests of the tod2map precision variants (float atomics, compensated float flush, float64 map)
against the FP64 oracle (reference_tod2map<double> semantics on the float32 inputs widened).

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
    the FP64 oracle over the whole TOD.  Bars: the north star's 1e-5 max relative error for the float
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
