"""This implementation against the reference's own GPU code, run on the same B200.

oracle/_ref/libgpu_mm_refgpu.so holds the reference's plan builder (PointingPrePlan.cu,
PointingPlan.cu with its CUB sort), its PointingPlanTester (PointingPlanTester.cu) and its planned
and unplanned operators (map2tod.cu, tod2map.cu, map2tod_unplanned.cu, tod2map_unplanned.cu),
compiled unchanged for sm_100a (oracle/Makefile).  The reference's own plan test (tests.py:227-254)
compares nmt_cumsum exactly and the plan as a multiset of its low 46 bits.  Here the comparison is
stricter: the reference's plan_mt, put in canonical (cell, cache line) order, must equal this
implementation's plan in all 64 bits, mflag and zflag included (the reference's within-cell order
is nondeterministic, the words themselves are not).  Operators agree within the float32 tolerances
of the other parity tests.
"""

import numpy as np
import pytest

import oracle
from tests._common import canonical, random_raster, rel_stats

pytestmark = pytest.mark.gpu

RL1_TOL = 1e-6
MAX_TOL = 1e-5


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    if not oracle.refgpu_available():
        pytest.skip("the reference-built comparator (oracle/_ref/libgpu_mm_refgpu.so) was not built")
    import gpu_mm_b200
    return gpu_mm_b200


def cases():
    rng = np.random.default_rng(2024)
    out = []
    for (ny, nx, periodic, ndet, nt, speed) in [(300, 500, True, 8, 4096, 0.7), (300, 500, False, 8, 4096, 0.9),
                                                (130, 1000, True, 16, 2048, 1.0), (64, 64, True, 4, 1024, 0.3),
                                                (200, 90, True, 4, 1024, 2.5), (1024, 2048, True, 64, 2048, 0.5)]:
        out.append((f"raster-{ny}x{nx}-{'p' if periodic else 'np'}-{speed}",
                    random_raster(rng, ndet, nt, ny, nx, periodic, speed=speed), ny, nx, periodic))
    # Scattered pointing: up to ~100 cells per cache line.
    n = 32 * 512
    xp = np.stack([rng.uniform(0, 639, n), rng.uniform(-700, 1400, n), rng.uniform(0, 7, n)]).astype(np.float32)
    out.append(("scattered", xp, 640, 700, True))
    return out


CASES = cases()


@pytest.mark.parametrize("i", range(len(CASES)), ids=[c[0] for c in CASES])
def test_plan_equals_reference_pointingplan(g, i):
    import torch
    _, xp, ny, nx, periodic = CASES[i]
    xg = torch.from_numpy(np.ascontiguousarray(xp)).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    ref = oracle.RefGpuPlan(xg, ny, nx, periodic)
    for k in ("plan_nmt", "ncl_per_threadblock", "planner_nblocks", "nmt_per_threadblock", "pointing_nblocks"):
        assert getattr(pp, k) == getattr(ref, k), k
    assert pp.overhead == pytest.approx(ref.overhead, rel=1e-12)
    ref_mt, ref_cs = ref.get()
    np.testing.assert_array_equal(pp.get_nmt_cumsum(), ref_cs)
    mt = plan.get_plan_mt()
    # The reference sorts by the 20 cell bits only: within a cell its order is whatever the chunk claims gave.
    assert np.all(np.diff((ref_mt & np.uint64(0xFFFFF)).astype(np.int64)) >= 0)
    np.testing.assert_array_equal(mt, canonical(ref_mt))


@pytest.mark.parametrize("i", [0, 2, 6])
def test_plan_equals_reference_plan_tester(g, i):
    """PointingPlanTester (the reference's simple per-line plan) gives the same nmt_cumsum and the same
    words on bits 0-45 (its mflag/zflag are not set, PointingPlanTester.cu:150)."""
    import torch
    _, xp, ny, nx, periodic = CASES[i]
    xg = torch.from_numpy(np.ascontiguousarray(xp)).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    t_mt, t_cs = oracle.refgpu_plan_tester(xg, ny, nx, periodic, capacity=pp.plan_nmt)
    np.testing.assert_array_equal(pp.get_nmt_cumsum(), t_cs[:pp.planner_nblocks])
    low = np.uint64((1 << 46) - 1)
    np.testing.assert_array_equal(np.sort(plan.get_plan_mt() & low), np.sort(t_mt & low))


@pytest.mark.parametrize("i", [0, 1, 4, 5])
def test_operators_equal_reference_gpu(g, i):
    """Planned and unplanned map2tod / tod2map against the reference's own GPU kernels."""
    import torch
    _, xp, ny, nx, periodic = CASES[i]
    rng = np.random.default_rng(7 + i)
    xg = torch.from_numpy(np.ascontiguousarray(xp)).cuda()
    pp = g.PointingPrePlan(xg, ny, nx, periodic_xcoord=periodic)
    plan = g.PointingPlan(pp, xg)
    ref = oracle.RefGpuPlan(xg, ny, nx, periodic)
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    offs_gpu = torch.from_numpy(lp_o.cell_offsets).cuda()
    nsamp = xg.numel() // 3
    m = torch.from_numpy(rng.standard_normal(3 * lp.npix).astype(np.float32)).cuda()
    t0 = torch.from_numpy(rng.standard_normal(nsamp).astype(np.float32)).cuda()
    errflags = torch.zeros(2048, dtype=torch.int32, device="cuda")
    for accum in (False, True):
        want = t0.clone()
        ref.map2tod(want, m, xg, lp_o, offs_gpu, accum=accum)
        got = t0.clone().reshape(xg.shape[1:])
        g.map2tod(got, g.LocalMap(lp, m), xg, plan, accum=accum)
        rl1, mx = rel_stats(got.cpu().numpy(), want.cpu().numpy())
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("planned map2tod", accum, rl1, mx)
        want_u = t0.clone()
        oracle.refgpu_unplanned_map2tod(want_u, m, xg, lp_o, offs_gpu, errflags, accum=accum)
        rl1, mx = rel_stats(want_u.cpu().numpy(), want.cpu().numpy())
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("reference planned vs unplanned", rl1, mx)
    t = torch.from_numpy(rng.standard_normal(nsamp).astype(np.float32)).cuda()
    want = torch.zeros(3 * lp.npix, device="cuda")
    ref.tod2map(want, t, xg, lp_o, offs_gpu)
    want_u = torch.zeros(3 * lp.npix, device="cuda")
    oracle.refgpu_unplanned_tod2map(want_u, t, xg, lp_o, offs_gpu, errflags)
    for pl in (plan, None):
        out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
        g.tod2map(out, t.reshape(xg.shape[1:]), xg, pl)
        for w, name in ((want, "planned"), (want_u, "unplanned")):
            rl1, mx = rel_stats(out.arr.cpu().numpy(), w.cpu().numpy())
            assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, name, rl1, mx)
