"""GPU tests of batches of TODs (gpu_mm_b200.TodBatch): one plan and one launch per operator for
many TODs, checked against the single-TOD planned path (plan contents, map2tod bit for bit, tod2map
within the float tolerance) and the oracle, plus CUDA-graph replay, error reporting and the
autotuner."""

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


def make_batch_inputs(seed, ny=256, nx=512, periodic=True, ntod=6):
    rng = np.random.default_rng(seed)
    sizes = [(int(rng.integers(1, 9)), 32 * int(rng.integers(8, 80))) for _ in range(ntod)]
    xps = [random_raster(rng, nd, nt, ny, nx, periodic, speed=float(rng.uniform(0.3, 1.2))) for nd, nt in sizes]
    tods = [rng.standard_normal(x.shape[1:]).astype(np.float32) for x in xps]
    return rng, xps, tods


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def owner_words(batch):
    import torch
    n = batch.total_lines
    return batch.plan[:8 * n].view(torch.int64).cpu().numpy().view(np.uint64)


def cellmap_bits(batch):
    off = ((8 * batch.total_lines + 127) // 128) * 128
    return batch.plan[off:off + (1 << 17)].cpu().numpy()


@pytest.mark.parametrize("periodic", [True, False])
def test_batch_plan_matches_single_plans(g, periodic):
    import torch
    ny, nx = 256, 512
    rng, xps, tods = make_batch_inputs(11 + periodic, ny, nx, periodic)
    xg = [cuda(x) for x in xps]
    tg = [cuda(t) for t in tods]
    lp = g.LocalPixelization.make_rectangle(ny, nx, periodic)
    b = g.TodBatch(xg, tg, lp)
    b.build_plan()
    b.check()
    got = owner_words(b)
    want, cells = [], set()
    for i, x in enumerate(xg):
        pp = g.PointingPrePlan(x, ny, nx, periodic_xcoord=periodic)
        plan = g.PointingPlan(pp, x)
        ow = plan._get_owner_mt() & np.uint64((1 << 47) - 1)
        want.append(ow | np.uint64(i << 48))
        cells |= set(int(c) for c in np.unique(plan.get_plan_mt() & np.uint64(0xFFFFF)))
    want = np.concatenate(want)
    # Sorted by cell, stable: (cell, tod, line) order.
    order = np.lexsort(((want >> np.uint64(20)) & np.uint64((1 << 26) - 1), want >> np.uint64(48),
                        want & np.uint64(0xFFFFF)))
    np.testing.assert_array_equal(got, want[order])
    bits = np.zeros(1 << 17, np.uint8)
    for c in cells:
        bits[c >> 3] |= np.uint8(1 << (c & 7))
    np.testing.assert_array_equal(cellmap_bits(b), bits)


def test_batch_operators_match_single_path(g):
    import torch
    ny, nx = 256, 512
    rng, xps, tods = make_batch_inputs(21, ny, nx, True)
    xg = [cuda(x) for x in xps]
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    lmap = g.LocalMap(lp, cuda(m))
    for accum in (False, True):
        t0 = [rng.standard_normal(x.shape[1:]).astype(np.float32) for x in xps]
        outs = [cuda(t) for t in t0]
        b = g.TodBatch(xg, outs, lp)
        b.build_plan()
        b.map2tod(lmap, accum=accum)
        b.check()
        for i, x in enumerate(xg):
            single = cuda(t0[i])
            pp = g.PointingPrePlan(x, ny, nx)
            g.map2tod(single, lmap, x, g.PointingPlan(pp, x), accum=accum)
            np.testing.assert_array_equal(outs[i].cpu().numpy(), single.cpu().numpy())
    tin = [cuda(t) for t in tods]
    b = g.TodBatch(xg, tin, lp)
    b.build_plan()
    out = g.LocalMap(lp, cuda(np.zeros(3 * lp.npix, np.float32)))
    b.tod2map(out)
    b.check()
    want = np.zeros(3 * lp.npix, np.float32)
    for x, t in zip(xps, tods):
        oracle.tod2map(want, t, x, lp_o)
    rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_batch_graph_replay_and_with_tods(g):
    import torch
    ny, nx = 256, 512
    rng, xps, tods = make_batch_inputs(31, ny, nx, True)
    xg = [cuda(x) for x in xps]
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lmap = g.LocalMap(lp, cuda(rng.standard_normal(3 * lp.npix).astype(np.float32)))
    outs = [torch.zeros(x.shape[1:], device="cuda") for x in xps]
    b = g.TodBatch(xg, outs, lp)
    b.build_plan()
    b.map2tod(lmap)
    torch.cuda.synchronize()
    eager = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    graph = b.capture(lambda s: (b.build_plan(s), b.map2tod(lmap, stream=s)))
    for o in outs:
        o.zero_()
    graph.replay()
    torch.cuda.synchronize()
    b.check()
    for o, e in zip(outs, eager):
        assert torch.equal(o, e)
    # Same pointing, other TOD arrays, same plan.
    tin = [cuda(t) for t in tods]
    b2 = b.with_tods(tin)
    out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    g2 = b2.capture(lambda s: b2.tod2map(out, stream=s))
    out.arr.zero_()
    g2.replay()
    torch.cuda.synchronize()
    b2.check()
    want = np.zeros(3 * lp.npix, np.float32)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    for x, t in zip(xps, tods):
        oracle.tod2map(want, t, x, lp_o)
    rl1, mx = rel_stats(out.arr.cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)
    del graph, g2


def test_batch_errors(g):
    import torch
    ny, nx = 128, 256
    rng, xps, tods = make_batch_inputs(41, ny, nx, True, ntod=3)
    xps[1] = xps[1].copy()
    xps[1][0, 0, 5] = ny + 3.0            # bad y in the second TOD
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    b = g.TodBatch([cuda(x) for x in xps], [cuda(t) for t in tods], lp)
    b.build_plan()
    with pytest.raises(RuntimeError, match="y"):
        b.check()
    # Descriptors that disagree with the batch's line count are reported, and nothing is read
    # outside the TODs (the owner kernel and the operators check every line against its TOD).
    rng, xps, tods = make_batch_inputs(42, ny, nx, True, ntod=3)
    b = g.TodBatch([cuda(x) for x in xps], [cuda(t) for t in tods], lp)
    d = b.descs.cpu().numpy().view(np.dtype([("xpointing", "<u8"), ("tod", "<u8"), ("nsamp", "<i8"), ("line0", "<i8")]))
    d["line0"][2] += 7
    b.descs.copy_(torch.from_numpy(d.view(np.uint8)))
    b.build_plan()
    with pytest.raises(RuntimeError):
        b.check()
    with pytest.raises(RuntimeError):
        g.TodBatch([cuda(xps[0])], [cuda(np.zeros(5, np.float32))], lp)


def test_autotune_small(g):
    import torch
    ny, nx = 256, 512
    rng, xps, tods = make_batch_inputs(51, ny, nx, True)
    xg = [cuda(x) for x in xps]
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lmap = g.LocalMap(lp, cuda(rng.standard_normal(3 * lp.npix).astype(np.float32)))
    outs = [torch.zeros(x.shape[1:], device="cuda") for x in xps]
    b = g.TodBatch(xg, outs, lp)
    scratch = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    best, times = g.autotune.autotune(b, lmap, scratch, candidates=[(4, 2, 64), (8, 4, 256)], reps=1)
    assert best in [(4, 2, 64), (8, 4, 256)] and len(times) == 2
    b.map2tod(lmap)
    b.check()
    for i, x in enumerate(xg):
        single = torch.zeros(x.shape[1:], device="cuda")
        pp = g.PointingPrePlan(x, ny, nx)
        g.map2tod(single, lmap, x, g.PointingPlan(pp, x))
        assert torch.equal(single, outs[i])


def test_build_plans_each_matches_single_builds(g):
    """build_plans_each (one owner pass, one sort by (TOD, cell), one scatter) gives each TOD the plan
    a batch of that one TOD builds, and merging those plans gives the batch's own plan."""
    import torch
    ny, nx = 256, 512
    rng, xps, tods = make_batch_inputs(61, ny, nx, True, ntod=7)
    xg = [cuda(x) for x in xps]
    tg = [cuda(t) for t in tods]
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    builder = g.TodBatch(xg, tg, lp, plan_buffers=False)
    singles = builder.build_plans_each()
    builder.check()
    for x, t, sp in zip(xg, tg, singles):
        one = g.TodBatch([x], [t], lp)
        one.build_plan()
        one.check()
        n = one.total_lines
        np.testing.assert_array_equal(sp.plan[:8 * n].cpu().numpy(), one.plan[:8 * n].cpu().numpy())
        np.testing.assert_array_equal(cellmap_bits(sp), cellmap_bits(one))
    b = g.TodBatch(xg, tg, lp)
    b.build_plan()
    want = owner_words(b)
    b.merge_plans(singles)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(owner_words(b), want)
