"""GPU tests at the full size of the large raster workload: 1024 detectors (32x32, 2 px spacing) x
2^18 samples (nsamp = 2^28), x sweep 0.7 px/sample over a periodic 3x8192x32768 map, LocalPixelization
holding the hit cells.

  * The plan equals the oracle's in every 64-bit word (plan_mt and the owner list), together with
    nmt_cumsum and the preplan geometry; and it equals the reference's own PointingPlan, built by the
    reference's code on the same GPU, put in canonical order (where that comparator was built).
  * Planned and unplanned map2tod and tod2map (both tod2map kernels) over the whole TOD agree with
    the multithreaded oracle (the reference's CPU operator arithmetic), and with the reference's own
    GPU operators where built.
  * The plan is deterministic (a second build gives the same words), planned map2tod is the same on
    every call of a plan-reuse loop (ten calls), and the operators are adjoint:
    <t, A m> = <A^T t, m> (A = map2tod), summed in float64.
  * At nsamp = 2^31, the largest the API accepts, planned and unplanned operators agree and the last
    detectors match the oracle.

Tolerances as in the parity tests: rel-L1 < 1e-6 and max|a-b| / max|b| < 1e-5; the adjoint identity
to 1e-6 of sum |t_i (A m)_i|.
"""

import ctypes
import os

import numpy as np
import pytest

import oracle
from tests._common import canonical, rel_stats

pytestmark = pytest.mark.gpu

RL1_TOL = 1e-6
MAX_TOL = 1e-5
NY, NX = 8192, 32768


@pytest.fixture(scope="module")
def workload():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    xp = synthetic.config2_xpointing(device="cuda")
    assert xp.shape == (3, 1024, 2 ** 18)
    pp = g.PointingPrePlan(xp, NY, NX)
    plan = g.PointingPlan(pp, xp)
    cells = synthetic.cells_of_plan(plan.get_plan_mt())
    lp = g.LocalPixelization.make_cells(NY, NX, cells)
    gen = torch.Generator(device="cuda").manual_seed(2028)
    m = torch.randn(3 * lp.npix, generator=gen, device="cuda")
    t = torch.randn(xp.shape[1:], generator=gen, device="cuda")
    return g, xp, pp, plan, lp, m, t


def gpu_rel_stats(a, b, chunk=1 << 26):
    """rel-L1 and max relative difference of two CUDA arrays, in float64 on the device, a chunk of
    elements at a time (so that 2^31-element arrays need no full-size float64 copies)."""
    a, b = a.reshape(-1), b.reshape(-1)
    dsum = asum = dmax = bmax = 0.0
    for i in range(0, a.numel(), chunk):
        ac, bc = a[i:i + chunk].double(), b[i:i + chunk].double()
        d = (ac - bc).abs()
        dsum += float(d.sum())
        asum += float(ac.abs().sum() + bc.abs().sum())
        dmax = max(dmax, float(d.max()))
        bmax = max(bmax, float(bc.abs().max()))
    return dsum / asum, dmax / bmax


@pytest.fixture(scope="module")
def host_inputs(workload):
    """Host copies of the workload (3 GiB of xpointing) and the oracle's view of the pixelization."""
    g, xp, pp, plan, lp, m, t = workload
    xs = xp.cpu().numpy()
    lp_o = oracle.Lpix(NY, NX, lp.cell_offsets_cpu, lp.ystride, lp.polstride, True)
    return xs, lp_o, m.cpu().numpy(), t.cpu().numpy()


def test_plan_equals_oracle_and_reference(workload, host_inputs):
    g, xp, pp, plan, lp, m, t = workload
    xs, lp_o, _, _ = host_inputs
    ref = oracle.preplan(xs, NY, NX, True)
    assert pp.plan_nmt == ref["nmt"]
    for k in ("ncl_per_threadblock", "planner_nblocks", "nmt_per_threadblock", "pointing_nblocks"):
        assert getattr(pp, k) == ref[k], k
    np.testing.assert_array_equal(pp.get_nmt_cumsum(), ref["nmt_cumsum"][:pp.planner_nblocks])
    mt_ref, owner_bits, err = oracle.plan(xs, NY, NX, True, nmt=ref["nmt"])
    assert err == 0
    mt = plan.get_plan_mt()
    np.testing.assert_array_equal(mt, mt_ref)
    owner = oracle.owner_words(xs, NY, mt_ref, owner_bits)
    np.testing.assert_array_equal(plan._get_owner_mt(), owner)
    bw = plan._get_band_words()
    np.testing.assert_array_equal(bw, oracle.band_words(xs, NY, NX, True, owner))
    assert np.mean(bw != 0) > 0.99        # the raster's lines take the band path
    if oracle.refgpu_available():
        rp = oracle.RefGpuPlan(xp, NY, NX, True)
        assert rp.plan_nmt == pp.plan_nmt
        rmt, rcs = rp.get()
        del rp
        np.testing.assert_array_equal(rcs, pp.get_nmt_cumsum())
        np.testing.assert_array_equal(canonical(rmt), mt)


def test_operators_equal_oracle(workload, host_inputs):
    """The whole TOD and map, planned and unplanned, both tod2map kernels, against the multithreaded
    oracle; and against the reference's own GPU operators where that comparator was built."""
    import torch
    g, xp, pp, plan, lp, m, t = workload
    xs, lp_o, m_h, t_h = host_inputs
    nthreads = os.cpu_count() or 1
    want = np.zeros(t_h.shape, np.float32)
    assert oracle.map2tod_mt(want, m_h, xs, lp_o, nthreads) == 0
    lmap = g.LocalMap(lp, m)
    tod = torch.empty(xp.shape[1:], device="cuda")
    for pl in (plan, None):
        g.map2tod(tod, lmap, xp, pl)
        rl1, mx = rel_stats(tod.cpu().numpy(), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("map2tod", pl is None, rl1, mx)
    want_m = np.zeros(3 * lp.npix, np.float32)
    assert oracle.tod2map_mt(want_m, t_h, xs, lp_o, nthreads) == 0
    lib = ctypes.CDLL(g.library_path())
    old = lib.gmm_get_planned_tod2map_kernel()
    try:
        for pl, which in ((plan, 0), (plan, 1), (None, 0)):
            lib.gmm_set_planned_tod2map_kernel(which)
            out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
            g.tod2map(out, t, xp, pl)
            rl1, mx = rel_stats(out.arr.cpu().numpy(), want_m)
            assert rl1 < RL1_TOL and mx < MAX_TOL, ("tod2map", pl is None, which, rl1, mx)
    finally:
        lib.gmm_set_planned_tod2map_kernel(old)
    if oracle.refgpu_available():
        rp = oracle.RefGpuPlan(xp, NY, NX, True)
        offs_gpu = torch.from_numpy(np.ascontiguousarray(lp_o.cell_offsets)).cuda()
        rt = torch.empty(xp[0].numel(), device="cuda")
        rp.map2tod(rt, m, xp, lp_o, offs_gpu)
        rl1, mx = rel_stats(rt.cpu().numpy(), want.reshape(-1))
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("reference GPU map2tod", rl1, mx)
        rm = torch.zeros(3 * lp.npix, device="cuda")
        rp.tod2map(rm, t.reshape(-1), xp, lp_o, offs_gpu)
        rl1, mx = rel_stats(rm.cpu().numpy(), want_m)
        assert rl1 < RL1_TOL and mx < MAX_TOL, ("reference GPU tod2map", rl1, mx)


def test_plan_deterministic(workload):
    g, xp, pp, plan, lp, m, t = workload
    pp2 = g.PointingPrePlan(xp, NY, NX)
    assert pp2.plan_nmt == pp.plan_nmt
    np.testing.assert_array_equal(pp2.get_nmt_cumsum(), pp.get_nmt_cumsum())
    plan2 = g.PointingPlan(pp2, xp)
    np.testing.assert_array_equal(plan2.get_plan_mt(), plan.get_plan_mt())


def test_map2tod_reuse_unplanned_and_oracle_sample(workload):
    import torch
    g, xp, pp, plan, lp, m, t = workload
    lmap = g.LocalMap(lp, m)
    first = torch.empty(xp.shape[1:], device="cuda")
    g.map2tod(first, lmap, xp, plan)
    tod = torch.empty_like(first)
    for _ in range(10):
        g.map2tod(tod, lmap, xp, plan)
        assert torch.equal(tod, first)
    g.map2tod(tod, lmap, xp, None)
    rl1, mx = gpu_rel_stats(tod, first)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)

    # A sample of detectors (first, last, and two in between) against the oracle.
    dets = [0, 17, 611, 1023]
    xs = np.ascontiguousarray(xp[:, dets, :].cpu().numpy())
    lp_o = oracle.Lpix(NY, NX, lp.cell_offsets_cpu, lp.ystride, lp.polstride, True)
    want = np.zeros(xs.shape[1:], np.float32)
    err = oracle.map2tod(want, m.cpu().numpy(), xs, lp_o)
    assert err == 0
    rl1, mx = rel_stats(first[dets].cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_tod2map_planned_unplanned_and_adjoint(workload):
    import torch
    g, xp, pp, plan, lp, m, t = workload
    out_p = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    g.tod2map(out_p, t, xp, plan)
    out_u = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    g.tod2map(out_u, t, xp, None)
    rl1, mx = gpu_rel_stats(out_p.arr, out_u.arr)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)

    am = torch.empty(xp.shape[1:], device="cuda")
    g.map2tod(am, g.LocalMap(lp, m), xp, plan)
    lhs = float((t.double() * am.double()).sum())
    rhs = float((out_p.arr.double() * m.double()).sum())
    scale = float((t.double() * am.double()).abs().sum())
    assert abs(lhs - rhs) < 1e-6 * scale, (lhs, rhs, scale)


def test_largest_nsamp():
    """nsamp = 2^31, the largest the API accepts (8192 detectors x 2^18 samples, the same raster
    construction; a periodic 3x8192x32768 rectangle map): the last samples sit at the top of the
    32-bit sample index range.  Planned and unplanned operators agree, and the last two detectors'
    map2tod matches the oracle."""
    import torch
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    xp = synthetic.raster_xpointing(256, 32, 2 ** 18, 2.0, 0.7, NX, 100.0, 2.0e-4, device="cuda")
    assert xp[0].numel() == 2 ** 31
    plan = g.PointingPlan(g.PointingPrePlan(xp, NY, NX), xp)
    lp = g.LocalPixelization.make_rectangle(NY, NX, True)
    gen = torch.Generator(device="cuda").manual_seed(2031)
    m = torch.randn(3 * lp.npix, generator=gen, device="cuda")
    lmap = g.LocalMap(lp, m)
    tod_p = torch.empty(xp.shape[1:], device="cuda")
    g.map2tod(tod_p, lmap, xp, plan)
    tod_u = torch.empty_like(tod_p)
    g.map2tod(tod_u, lmap, xp, None)
    rl1, mx = gpu_rel_stats(tod_p, tod_u)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)
    del tod_u
    xs = np.ascontiguousarray(xp[:, -2:, :].cpu().numpy())
    want = np.zeros(xs.shape[1:], np.float32)
    assert oracle.map2tod(want, m.cpu().numpy(), xs, oracle.Lpix.rectangle(NY, NX, True)) == 0
    rl1, mx = rel_stats(tod_p[-2:].cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)
    t = tod_p
    t.normal_(generator=gen)
    out_p = torch.zeros(3 * lp.npix, device="cuda")
    g.tod2map(g.LocalMap(lp, out_p), t, xp, plan)
    out_u = torch.zeros(3 * lp.npix, device="cuda")
    g.tod2map(g.LocalMap(lp, out_u), t, xp, None)
    rl1, mx = gpu_rel_stats(out_p, out_u)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)
