"""GPU parity tests: the sm_100a path (through the drop-in Python API and through the C ABI) against
the oracle, on the reference's own golden vectors and on seeded synthetic scans.

Tolerances (float32 operators): rel-L1 = sum|a-b| / (sum|a|+sum|b|) < 1e-6, the reference's metric
(tests.py:220-224, :277, :326), and max|a-b| / max|b| < 1e-5.  Plans are compared bit for bit.
"""

import ctypes

import numpy as np
import pytest

import oracle
from tests._common import random_raster, rel_stats

pytestmark = pytest.mark.gpu

RL1_TOL = 1e-6
MAX_TOL = 1e-5


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200
    return gpu_mm_b200


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def host(t):
    return t.detach().cpu().numpy()


def build_plan(g, xp_gpu, ny, nx, periodic):
    pp = g.PointingPrePlan(xp_gpu, ny, nx, periodic_xcoord=periodic)
    return pp, g.PointingPlan(pp, xp_gpu)


def check_plan(g, xp, ny, nx, periodic, pp, plan):
    ref = oracle.preplan(xp, ny, nx, periodic)
    assert pp.plan_nmt == ref["nmt"]
    for k in ("ncl_per_threadblock", "planner_nblocks", "nmt_per_threadblock", "pointing_nblocks"):
        assert getattr(pp, k) == ref[k], k
    np.testing.assert_array_equal(pp.get_nmt_cumsum(), ref["nmt_cumsum"][:pp.planner_nblocks])
    mt_ref, owner_ref, err = oracle.plan(xp, ny, nx, periodic, nmt=ref["nmt"])
    assert err == 0
    mt = plan.get_plan_mt()
    np.testing.assert_array_equal(mt, mt_ref)   # all 64 bits, canonical order
    owner = oracle.owner_words(xp, ny, mt_ref, owner_ref)
    np.testing.assert_array_equal(plan._get_owner_mt(), owner)
    np.testing.assert_array_equal(plan._get_band_words(), oracle.band_words(xp, ny, nx, periodic, owner))


def lpix_from(g, ny, nx, offs, ys, ps, periodic):
    return g.LocalPixelization(ny, nx, offs, ys, ps, periodic)


GOLDEN = ("wrap_rect", "flat_cells_accum", "partial_missing", "scattered")


@pytest.mark.parametrize("name", GOLDEN)
def test_golden_vectors(g, golden_ops, name):
    """Planned and unplanned operators reproduce the reference header's outputs (golden vectors)."""
    p = golden_ops[f"{name}__params"]
    ny, nx, periodic, ys, ps, partial, accum = (int(p[0]), int(p[1]), bool(p[2]), int(p[3]), int(p[4]),
                                                bool(p[5]), bool(p[6]))
    xp = golden_ops[f"{name}__xpointing"]
    lp = lpix_from(g, ny, nx, golden_ops[f"{name}__cell_offsets"], ys, ps, periodic)
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, periodic)
    check_plan(g, xp, ny, nx, periodic, pp, plan)
    lmap = g.LocalMap(lp, cuda(golden_ops[f"{name}__map"].astype(np.float32)))
    want = golden_ops[f"{name}__m2t_out"]
    for pl in (plan, None):
        tod = cuda(golden_ops[f"{name}__tod_init"].astype(np.float32))
        g.map2tod(tod, lmap, xg, pl, partial_pixelization=partial, accum=accum)
        rl1, mx = rel_stats(host(tod), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)
    want = golden_ops[f"{name}__t2m_out"]
    for pl in (plan, None):
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, cuda(golden_ops[f"{name}__tod_in"].astype(np.float32)), xg, pl, partial_pixelization=partial)
        rl1, mx = rel_stats(host(out.arr), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)


def test_golden_errors(g, golden_ops):
    """Out-of-range y/x raise the reference's messages (check_arguments.cu:48-51), in the preplan
    and in the unplanned operators."""
    name = "errors"
    p = golden_ops[f"{name}__params"]
    ny, nx = int(p[0]), int(p[1])
    xg = cuda(golden_ops[f"{name}__xpointing"])
    with pytest.raises(RuntimeError, match="y-value is outside range"):
        g.PointingPrePlan(xg, ny, nx, periodic_xcoord=False)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    lmap = g.LocalMap(lp, cuda(golden_ops[f"{name}__map"].astype(np.float32)))
    tod = cuda(np.zeros(golden_ops[f"{name}__tod_in"].shape, np.float32))
    with pytest.raises(RuntimeError, match="y-value is outside range"):
        g.map2tod(tod, lmap, xg, None)


SYNTH = [
    # (ny, nx, periodic, ndet, nt, speed, seed)
    (300, 500, True, 8, 4096, 0.7, 0),
    (300, 500, False, 8, 4096, 0.9, 1),
    (130, 1000, True, 16, 2048, 1.0, 2),     # fast scan: lines span up to 33 px
    (64, 64, True, 4, 1024, 0.3, 3),         # one cell, wrap inside it
    (200, 90, True, 4, 1024, 2.5, 4),        # narrow map: x wraps every ~36 samples
]


@pytest.mark.parametrize("case", SYNTH)
def test_synthetic_scans(g, case):
    ny, nx, periodic, ndet, nt, speed, seed = case
    rng = np.random.default_rng(1000 + seed)
    xp = random_raster(rng, ndet, nt, ny, nx, periodic, speed=speed)
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, periodic)
    check_plan(g, xp, ny, nx, periodic, pp, plan)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    lmap = g.LocalMap(lp, cuda(m))
    for accum in (False, True):
        t0 = rng.standard_normal(xp.shape[1:]).astype(np.float32)
        want = t0.copy()
        oracle.map2tod(want, m, xp, lp_o, False, accum)
        for pl in (plan, None):
            tod = cuda(t0)
            g.map2tod(tod, lmap, xg, pl, accum=accum)
            rl1, mx = rel_stats(host(tod), want)
            assert rl1 < RL1_TOL and mx < MAX_TOL, (accum, pl is None, rl1, mx)
    t = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    m0 = rng.standard_normal(3 * lp.npix).astype(np.float32)
    want = m0.copy()
    oracle.tod2map(want, t, xp, lp_o)
    for pl in (plan, None):
        out = g.LocalMap(lp, cuda(m0))
        g.tod2map(out, cuda(t), xg, pl)
        rl1, mx = rel_stats(host(out.arr), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)


def test_partial_pixelization_and_missing_cells(g):
    """Cells absent from the local map read as zero with partial_pixelization, and raise without it
    (map2tod.cu:127-129, gpu_mm_internals.hpp:280)."""
    rng = np.random.default_rng(77)
    ny, nx = 256, 320
    xp = random_raster(rng, 8, 2048, ny, nx, True, speed=0.8)
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, True)
    nyc, nxc = 4, 5
    present = np.ones((nyc, nxc), bool)
    present[1, 2] = present[2, 0] = present[0, 4] = False
    offs = np.full((nyc, nxc), -1, np.int64)
    k = 0
    for iy in range(nyc):
        for ix in range(nxc):
            if present[iy, ix]:
                offs[iy, ix] = 3 * 4096 * k
                k += 1
    lp = g.LocalPixelization(ny, nx, offs, 64, 4096, True)
    lp_o = oracle.Lpix(ny, nx, offs, 64, 4096, True)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    lmap = g.LocalMap(lp, cuda(m))
    want = np.zeros(xp.shape[1:], np.float32)
    err = oracle.map2tod(want, m, xp, lp_o, False, False)   # same values as partial=True, plus the error bit
    assert err & oracle.ERR_NOT_IN_PIXELIZATION   # the scan does touch a missing cell
    for pl in (plan, None):
        tod = cuda(np.zeros(xp.shape[1:], np.float32))
        g.map2tod(tod, lmap, xg, pl, partial_pixelization=True)
        rl1, mx = rel_stats(host(tod), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL
        with pytest.raises(RuntimeError, match="not in LocalPixelization"):
            g.map2tod(tod, lmap, xg, pl, partial_pixelization=False)
    t = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, t, xp, lp_o, True)
    for pl in (plan, None):
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, cuda(t), xg, pl, partial_pixelization=True)
        rl1, mx = rel_stats(host(out.arr), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL
        with pytest.raises(RuntimeError, match="not in LocalPixelization"):
            g.tod2map(out, cuda(t), xg, pl, partial_pixelization=False)


@pytest.mark.parametrize("ndet,nt", [(8, 2048), (6, 1056), (96, 24)])
def test_response_variants(g, ndet, nt):
    """Per-detector (T, P) response (map2tod_response.cu, tod2map_response.cu), as in tests.py:295-354;
    detector lengths that are a power of two, not a power of two, and shorter than a cache line."""
    rng = np.random.default_rng(31 + ndet)
    ny, nx = 200, 400
    xp = random_raster(rng, ndet, nt, ny, nx, True)
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, True)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    resp = rng.uniform(0.5, 2.0, (2, ndet)).astype(np.float32)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    for accum in (False, True):
        t0 = rng.standard_normal((ndet, nt)).astype(np.float32)
        want = t0.copy()
        oracle.response_map2tod(want, m, xp, resp, lp_o, False, accum)
        tod = cuda(t0)
        g.map2tod(tod, g.LocalMap(lp, cuda(m)), xg, plan, response=cuda(resp), accum=accum)
        rl1, mx = rel_stats(host(tod), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL
    t = rng.standard_normal((ndet, nt)).astype(np.float32)
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.response_tod2map(want, t, xp, resp, lp_o)
    out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
    g.tod2map(out, cuda(t), xg, plan, response=cuda(resp))
    rl1, mx = rel_stats(host(out.arr), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL


def test_config1_full_size(g):
    """The small benchmark configuration (2^22 samples, 3x1024x2048 map) end to end against the oracle."""
    from gpu_mm_b200 import synthetic
    c = synthetic.config1(device="cpu")
    xp = c["xpointing"].numpy()
    ny, nx = c["nypix"], c["nxpix"]
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, True)
    check_plan(g, xp, ny, nx, True, pp, plan)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = c["map"].numpy().reshape(-1)
    want = np.zeros(xp.shape[1:], np.float32)
    oracle.map2tod(want, m, xp, lp_o)
    lmap = g.LocalMap(lp, cuda(m))
    for pl in (plan, None):
        tod = cuda(np.zeros(xp.shape[1:], np.float32))
        g.map2tod(tod, lmap, xg, pl)
        rl1, mx = rel_stats(host(tod), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)
    t = c["tod"].numpy()
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, t, xp, lp_o)
    for pl in (plan, None):
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, cuda(t), xg, pl)
        rl1, mx = rel_stats(host(out.arr), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)


def test_aligned_and_unaligned_arrays(g):
    """The planned operators have a 16-byte-load kernel (xpointing and TOD 16-byte aligned) and a
    one-sample-per-lane kernel for other alignments.  Both must match the oracle, and map2tod must
    give the same bits through either, and through the unplanned operator (each sample is evaluated
    with the same explicitly rounded operations)."""
    import torch
    rng = np.random.default_rng(77)
    ny, nx, periodic = 512, 1024, True
    ndet, nt = 12, 4096
    xp = random_raster(rng, ndet, nt, ny, nx, periodic, speed=0.6)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    t = rng.standard_normal((ndet, nt)).astype(np.float32)
    lmap = g.LocalMap(lp, cuda(m))
    want_tod = np.zeros((ndet, nt), np.float32)
    oracle.map2tod(want_tod, m, xp, lp_o, False, False)
    want_map = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want_map, t, xp, lp_o)

    def offset_copy(a, off):
        flat = torch.zeros(a.size + off, dtype=torch.float32, device="cuda")
        v = flat[off:].view(a.shape)
        v.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        return v

    tods = []
    for off in (0, 1):
        xg = offset_copy(xp, off)
        assert (xg.data_ptr() % 16 == 0) == (off == 0)
        pp, plan = build_plan(g, xg, ny, nx, periodic)
        tod = offset_copy(np.zeros((ndet, nt), np.float32), off)
        g.map2tod(tod, lmap, xg, plan)
        rl1, mx = rel_stats(host(tod), want_tod)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (off, rl1, mx)
        tods.append(host(tod))
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, offset_copy(t, off), xg, plan)
        rl1, mx = rel_stats(host(out.arr), want_map)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (off, rl1, mx)
    np.testing.assert_array_equal(tods[0], tods[1])
    # The unplanned operator evaluates each sample with the same rounded operations.
    xg = offset_copy(xp, 0)
    tod = offset_copy(np.zeros((ndet, nt), np.float32), 0)
    g.map2tod(tod, lmap, xg, None)
    np.testing.assert_array_equal(host(tod), tods[0])


@pytest.mark.parametrize("periodic", [True, False])
def test_fast_and_general_paths(g, periodic):
    """The planned kernels take a branch-free path for a line (or group of lines) whose samples are all
    ordinary, and the general per-sample path otherwise.  Plant the cases the general path exists
    for: large angles (|2a| > 1024), periodic x that needs folding or lands on x = nx, y = ny-1 and
    non-periodic x = nx-2.  Both alignments; results against the oracle."""
    import torch
    rng = np.random.default_rng(5150 + periodic)
    ny, nx = 256, 512
    ndet, nt = 16, 2048
    xp = random_raster(rng, ndet, nt, ny, nx, periodic, speed=0.4)
    xp64 = xp.astype(np.float64)
    pick = lambda k: (rng.integers(0, ndet, k), rng.integers(0, nt, k))
    d, t = pick(40)
    xp64[2, d, t] = rng.choice([-600.0, 600.0, 5000.0], 40)
    d, t = pick(20)
    xp64[0, d, t] = ny - 1.0
    if periodic:
        d, t = pick(60)
        xp64[1, d, t] -= nx
        d, t = pick(60)
        xp64[1, d, t] = np.minimum(xp64[1, d, t] + nx, 2.0 * nx)
        d, t = pick(10)
        xp64[1, d, t] = float(nx)
    else:
        d, t = pick(20)
        xp64[1, d, t] = nx - 2.0
    xp = xp64.astype(np.float32)
    lp_o = oracle.Lpix.rectangle(ny, nx, periodic)
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    tv = rng.standard_normal((ndet, nt)).astype(np.float32)
    lmap = g.LocalMap(lp, cuda(m))
    want_tod = np.zeros((ndet, nt), np.float32)
    oracle.map2tod(want_tod, m, xp, lp_o, False, False)
    want_map = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want_map, tv, xp, lp_o)
    for off in (0, 1):
        flat = torch.zeros(xp.size + off, dtype=torch.float32, device="cuda")
        xg = flat[off:].view(xp.shape)
        xg.copy_(torch.from_numpy(xp))
        pp, plan = build_plan(g, xg, ny, nx, periodic)
        tflat = torch.zeros(tv.size + off, dtype=torch.float32, device="cuda")
        tod = tflat[off:].view(tv.shape)
        g.map2tod(tod, lmap, xg, plan)
        rl1, mx = rel_stats(host(tod), want_tod)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (off, rl1, mx)
        tod.copy_(torch.from_numpy(tv))
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, tod, xg, plan)
        rl1, mx = rel_stats(host(out.arr), want_map)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (off, rl1, mx)


def test_plan_reuse_and_buffers(g):
    """Caller-supplied buffers (gpu_mm.py:1253-1299): one shared tmp_buf for several plans; a plan is
    reusable across calls and gives identical results."""
    import torch
    rng = np.random.default_rng(8)
    ny, nx = 256, 256
    xps = [random_raster(rng, 4, 1024, ny, nx, True) for _ in range(3)]
    tmp_pp = torch.empty(1024, dtype=torch.int32, device="cuda")
    plans = []
    tmp = None
    for xp in xps:
        xg = cuda(xp)
        pp = g.PointingPrePlan(xg, ny, nx, buf=torch.empty(1024, dtype=torch.int32, device="cuda"), tmp_buf=tmp_pp)
        if tmp is None or tmp.numel() < pp.plan_constructor_tmp_nbytes:
            tmp = torch.empty(2 * pp.plan_constructor_tmp_nbytes, dtype=torch.uint8, device="cuda")
        plan = g.PointingPlan(pp, xg, buf=torch.empty(pp.plan_nbytes, dtype=torch.uint8, device="cuda"), tmp_buf=tmp)
        plans.append((xp, xg, pp, plan))
    for xp, xg, pp, plan in plans:
        check_plan(g, xp, ny, nx, True, pp, plan)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lmap = g.LocalMap(lp, cuda(rng.standard_normal(3 * lp.npix).astype(np.float32)))
    xp, xg, pp, plan = plans[0]
    outs = []
    for _ in range(3):
        tod = cuda(np.zeros(xp.shape[1:], np.float32))
        g.map2tod(tod, lmap, xg, plan)
        outs.append(host(tod))
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_dynamic_map(g):
    """DynamicMap grown chunk by chunk, randomly permuted and finalized equals the reference
    tod2map on a global map (tests.py:356-411)."""
    rng = np.random.default_rng(12)
    ny, nx = 300, 700
    xp = random_raster(rng, 4, 4096, ny, nx, True, speed=0.6)
    t = rng.standard_normal((4, 4096)).astype(np.float32)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    ref = np.zeros(3 * lp_o.npix, np.float32)
    oracle.tod2map(ref, t, xp, lp_o)
    nyc, nxc = lp_o.nycells, lp_o.nxcells
    ref_global = ref.reshape(3, 64 * nyc, 64 * nxc)[:, :ny, :nx]
    dmap = g.DynamicMap(ny, nx, np.float32, initial_ncells=1)
    for a, b in ((0, 1024), (1024, 1056), (1056, 4096)):
        xc = cuda(np.ascontiguousarray(xp[:, :, a:b]))
        pp = g.PointingPrePlan(xc, ny, nx)
        plan = g.PointingPlan(pp, xc)
        g.tod2map(dmap, cuda(np.ascontiguousarray(t[:, a:b])), xc, plan)
    dmap.randomly_permute()
    lmap = dmap.finalize()
    got = lmap.to_global()
    rl1, mx = rel_stats(got, ref_global)
    assert rl1 < RL1_TOL and mx < MAX_TOL


def test_dynamic_map_cell_mask_growth_and_errors(g):
    """A cell mask limits growth to the target cells (tod2map with partial_pixelization, as the
    reference requires); capacity grows from one cell; permute() rejects a cell list that is not the
    footprint; the map cannot grow after permute() or be finalized twice."""
    import torch
    rng = np.random.default_rng(33)
    ny, nx = 256, 512
    xp = random_raster(rng, 4, 2048, ny, nx, True, speed=0.8)
    t = rng.standard_normal((4, 2048)).astype(np.float32)
    nyc, nxc = 4, 8
    mask = np.zeros((nyc, nxc), bool)
    mask[:, ::2] = True
    mask[1, :] = True
    offs = np.full((nyc, nxc), -1, np.int64)
    for k, (iy, ix) in enumerate(zip(*np.nonzero(mask))):
        offs[iy, ix] = 3 * 4096 * k
    lp_o = oracle.Lpix(ny, nx, offs, 64, 4096, True)
    want = np.zeros(3 * lp_o.npix, np.float32)
    oracle.tod2map(want, t, xp, lp_o, True)
    xc = cuda(xp)
    plan = g.PointingPlan(g.PointingPrePlan(xc, ny, nx), xc)
    dmap = g.DynamicMap(ny, nx, np.float32, cell_mask=mask, initial_ncells=1)
    with pytest.raises(RuntimeError, match="have_cell_mask"):
        g.tod2map(dmap, cuda(t), xc, plan, partial_pixelization=False)
    g.tod2map(dmap, cuda(t), xc, plan, partial_pixelization=True)
    touched = {(int(c) >> 10, int(c) & 1023) for c in np.unique(plan.get_plan_mt() & np.uint64(0xFFFFF))}
    present = {c for c in touched if mask[c]}
    assert dmap.ncells_curr == len(present) and dmap.ncells_allocated >= dmap.ncells_curr
    iy, ix = np.nonzero(dmap._unstable_pixelization.cell_offsets_gpu.cpu().numpy() >= 0)
    assert set(zip(iy.tolist(), ix.tolist())) == present
    with pytest.raises(RuntimeError, match="do not match footprint"):
        dmap.permute(np.append(iy[:-1], iy[0]), np.append(ix[:-1], ix[0]))
    dmap.permute(iy[::-1].copy(), ix[::-1].copy())
    with pytest.raises(RuntimeError, match="after MpiPixelization"):
        dmap.expand(plan)
    lmap = dmap.finalize()
    with pytest.raises(RuntimeError, match="Double call"):
        dmap.finalize()
    got = lmap.to_global()
    ref_global = np.zeros((3, ny, nx), np.float32)
    for (cy, cx) in present:
        k = offs[cy, cx] // 4096
        blk = want.reshape(-1, 3, 64, 64)[k // 3]
        ref_global[:, 64 * cy:64 * cy + 64, 64 * cx:64 * cx + 64] = blk[:, :min(64, ny - 64 * cy), :min(64, nx - 64 * cx)]
    rl1, mx = rel_stats(got, ref_global)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_reference_cpu_operators(g):
    """plan='reference' runs the library's CPU operator and agrees with the oracle."""
    rng = np.random.default_rng(4)
    ny, nx = 100, 200
    xp = random_raster(rng, 2, 512, ny, nx, True)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    tod = np.zeros(xp.shape[1:], np.float32)
    g.map2tod(tod, g.LocalMap(lp, m), xp, 'reference')
    want = np.zeros_like(tod)
    oracle.map2tod(want, m, xp, lp_o)
    np.testing.assert_allclose(tod, want, rtol=1e-6, atol=1e-6)


def test_reference_enumerator_on_gpu(g):
    """The oracle's cell slots equal the reference's own device-only cell_enumerator, run on the GPU
    from oracle/_ref (skipped where that library was not built)."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    import torch
    rng = np.random.default_rng(21)
    for (ny, nx, periodic) in ((300, 400, True), (300, 400, False), (70, 64, True)):
        n = 8192
        xp = np.zeros((3, n), np.float32)
        xp[0] = rng.uniform(0, ny - 1, n)
        lo, hi = ((-nx, 2 * nx) if periodic else (0, nx - 2))
        xp[1] = rng.uniform(lo, hi, n)
        xp[1, :64] = np.clip(np.arange(64) * 64.0 - 1.0, lo, hi)
        xg = cuda(xp)
        slots = torch.zeros(6 * n, dtype=torch.int32, device="cuda")
        errs = torch.zeros(n, dtype=torch.int32, device="cuda")
        rc = oracle.ref().ref_enumerate_gpu(xg.data_ptr(), n, ny, nx, int(periodic), slots.data_ptr(), errs.data_ptr())
        assert rc == 0
        np.testing.assert_array_equal(host(slots).reshape(n, 6), oracle.sample_slots(xp, ny, nx, periodic))


def test_c_abi_direct(g):
    """Calls libgpu_mm_b200.so through ctypes with device pointers (the boundary a cgo/JNI/ctypes user
    binds), including the deferred error word."""
    import torch
    L = ctypes.CDLL(g.library_path())
    L.gmm_last_error.restype = ctypes.c_char_p

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

    rng = np.random.default_rng(2)
    ny, nx = 256, 512
    xp = random_raster(rng, 4, 2048, ny, nx, True)
    nsamp = xp.size // 3
    xg = cuda(xp)
    nmt = torch.zeros(1024, dtype=torch.int32, device="cuda")
    err = torch.zeros(1024, dtype=torch.int32, device="cuda")
    info = Info()
    rc = L.gmm_preplan(ctypes.c_void_p(xg.data_ptr()), ctypes.c_int64(nsamp), ny, nx, 1, ctypes.c_void_p(nmt.data_ptr()),
                       ctypes.c_void_p(err.data_ptr()), 0, None, ctypes.byref(info))
    assert rc == 0, L.gmm_last_error()
    buf = torch.empty(info.plan_nbytes, dtype=torch.uint8, device="cuda")
    tmp = torch.empty(info.plan_constructor_tmp_nbytes, dtype=torch.uint8, device="cuda")
    rc = L.gmm_plan_build(ctypes.byref(info), ctypes.c_void_p(nmt.data_ptr()), ctypes.c_void_p(xg.data_ptr()),
                          ctypes.c_void_p(buf.data_ptr()), ctypes.c_int64(buf.numel()), ctypes.c_void_p(tmp.data_ptr()),
                          ctypes.c_int64(tmp.numel()), 0, None)
    assert rc == 0, L.gmm_last_error()
    mt_ref, _, _ = oracle.plan(xp, ny, nx, True)
    np.testing.assert_array_equal(host(buf[:8 * info.plan_nmt].view(torch.int64)).view(np.uint64), mt_ref)

    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    offs = cuda(lp_o.cell_offsets)
    lp = Lpix(ny, nx, 1, lp_o.nycells, lp_o.nxcells, 0, lp_o.ystride, lp_o.polstride, lp_o.npix, offs.data_ptr())
    m = rng.standard_normal(3 * lp_o.npix).astype(np.float32)
    mg = cuda(m)
    tod = torch.zeros(nsamp, dtype=torch.float32, device="cuda")
    word = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.gmm_planned_map2tod(ctypes.c_void_p(tod.data_ptr()), ctypes.c_void_p(mg.data_ptr()),
                               ctypes.c_void_p(xg.data_ptr()), ctypes.byref(lp), ctypes.byref(info),
                               ctypes.c_void_p(buf.data_ptr()), 0, 0, ctypes.c_void_p(word.data_ptr()), None)
    assert rc == 0
    assert L.gmm_errword_read(ctypes.c_void_p(word.data_ptr()), 0, None) == 0
    want = np.zeros(nsamp, np.float32)
    oracle.map2tod(want, m, xp, lp_o)
    rl1, mx = rel_stats(host(tod), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL
    # Missing cells raise bit 8 through the deferred word.
    offs2 = np.full_like(lp_o.cell_offsets, -1)
    og = cuda(offs2)
    lp.cell_offsets = og.data_ptr()
    rc = L.gmm_planned_map2tod(ctypes.c_void_p(tod.data_ptr()), ctypes.c_void_p(mg.data_ptr()),
                               ctypes.c_void_p(xg.data_ptr()), ctypes.byref(lp), ctypes.byref(info),
                               ctypes.c_void_p(buf.data_ptr()), 0, 0, ctypes.c_void_p(word.data_ptr()), None)
    assert rc == 0
    assert L.gmm_errword_read(ctypes.c_void_p(word.data_ptr()), 0, None) == 8
    assert L.gmm_errword_read(ctypes.c_void_p(word.data_ptr()), 8, None) == 0


@pytest.mark.parametrize("periodic", [True, False])
def test_maximum_map_size(g, periodic):
    """The largest global map the API accepts (65536 x 65536 pixels, 1024 x 1024 cells), scanned
    next to its last row and column of cells: cell ids reach (1023, 1023), and with periodic x the
    scan wraps from column 65535 to column 0.  The local map holds only the hit cells.  Plans bit for
    bit, operators against the oracle."""
    ny = nx = 65536
    rng = np.random.default_rng(65536 + periodic)
    ndet, nt = 8, 1024
    t = np.arange(nt, dtype=np.float64)[None, :]
    d = np.arange(ndet, dtype=np.float64)[:, None]
    y = (ny - 6.0) - 0.013 * t - 2.0 * d
    if periodic:
        x = 65400.0 + 0.7 * t + 1.5 * d          # reaches 66126: folds onto columns 0..590
    else:
        x = 65533.0 - 0.7 * t - 1.5 * d          # down from the last valid column
    al = rng.uniform(-3.0, 3.0, (ndet, nt))
    xp = np.stack([y, x, al]).astype(np.float32)
    xg = cuda(xp)
    pp, plan = build_plan(g, xg, ny, nx, periodic)
    check_plan(g, xp, ny, nx, periodic, pp, plan)
    from gpu_mm_b200 import synthetic
    cells = synthetic.cells_of_plan(plan.get_plan_mt())
    assert (1023, 1023) in cells and (not periodic or (1023, 0) in cells), cells
    lp = g.LocalPixelization.make_cells(ny, nx, cells, periodic)
    lp_o = oracle.Lpix(ny, nx, lp.cell_offsets_cpu, lp.ystride, lp.polstride, periodic)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    want = np.zeros(xp.shape[1:], np.float32)
    assert oracle.map2tod(want, m, xp, lp_o) == 0
    lmap = g.LocalMap(lp, cuda(m))
    for pl in (plan, None):
        tod = cuda(np.zeros(xp.shape[1:], np.float32))
        g.map2tod(tod, lmap, xg, pl)
        rl1, mx = rel_stats(host(tod), want)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)
    tv = rng.standard_normal(xp.shape[1:]).astype(np.float32)
    want_m = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want_m, tv, xp, lp_o)
    for pl in (plan, None):
        out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
        g.tod2map(out, cuda(tv), xg, pl)
        rl1, mx = rel_stats(host(out.arr), want_m)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (pl is None, rl1, mx)
