"""GPU tests of the reference's test utilities, ToyPointing and PointingPlanTester, used the way the
reference's own plan test uses them (tests.py:119-254): a random ToyPointing, its preplan and plan,
and the tester's simple plan, which must hold the same (cell, cache line) pairs (bits 0-45) and the
same per-block cumulative counts."""

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

MASK46 = np.uint64((1 << 46) - 1)


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200
    return gpu_mm_b200


def toy_raster(nsamp, ny, nx, speed, total_drift):
    """ToyPointing's raster restated in Python (ToyPointing.cu:63-108), for a check of the C++ one."""
    drift = total_drift / (9.0 * nsamp)          # total_drift / (3 * xpointing size)
    out = np.zeros((3, nsamp), np.float32)
    y = x = 1.0
    vel = speed
    ylo, yhi = 1.1 * speed, ny - 2 - 1.1 * speed
    for s in range(nsamp):
        out[0, s], out[1, s], out[2, s] = y, x, 1.0
        if vel > 0 and y > yhi:
            vel = -speed
        if vel < 0 and y < ylo:
            vel = speed
        y += vel
        x += vel + drift
        if x < 0.0:
            x += nx
        if x > nx:
            x -= nx
    return out


def test_toy_pointing_raster(g):
    tp = g.ToyPointing(4, 8192, 300, 700, 0.37, 250.0, noisy=False)
    assert tp.xpointing_cpu.shape == (3, 4, 8192) and tuple(tp.xpointing_gpu.shape) == (3, 4, 8192)
    want = toy_raster(4 * 8192, 300, 700, 0.37, 250.0).reshape(3, 4, 8192)
    np.testing.assert_array_equal(tp.xpointing_cpu, want)
    np.testing.assert_array_equal(tp.xpointing_gpu.cpu().numpy(), want)
    assert tp.drift_speed == pytest.approx(250.0 / (9 * 4 * 8192))
    assert "ToyPointing(tod_shape=(4,8192)" in str(tp)
    with pytest.raises(RuntimeError):
        g.ToyPointing(None, 4096, 300, 700, 1.5, 250.0, noisy=False)      # scan_speed > 1


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_plan_tester_matches_plan(g, seed):
    np.random.seed(seed)
    tp = g.ToyPointing.make_random(1 << 18, noisy=False)
    xp = tp.xpointing_gpu
    pp = g.PointingPrePlan(xp, tp.nypix_global, tp.nxpix_global)
    plan = g.PointingPlan(pp, xp)
    pt = g.PointingPlanTester(pp, xp)
    assert (pt.nsamp, pt.plan_nmt, pt.planner_nblocks) == (pp.nsamp, pp.plan_nmt, pp.planner_nblocks)
    np.testing.assert_array_equal(pt.nmt_cumsum, pp.get_nmt_cumsum())
    # The plan (sorted by cell) and the tester (sorted by word) hold the same pairs.
    mt = np.sort(plan.get_plan_mt() & MASK46)
    np.testing.assert_array_equal(mt, pt.sorted_mt)
    # Pixel indices of a sample of the samples against the oracle's locate().
    flat = tp.xpointing_cpu.reshape(3, -1)
    for s in np.random.default_rng(seed).integers(0, pt.nsamp, 500):
        idx, _, err = oracle.locate(flat[0, s], flat[1, s], tp.nypix_global, tp.nxpix_global, True)
        assert err == 0 and (pt.iypix[s], pt.ixpix[s]) == (idx[0], idx[2])
