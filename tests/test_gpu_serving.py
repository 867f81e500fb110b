"""GPU tests of the serving loop (gpu_mm_b200.PointingServer): continuous batching of plan, map2tod
and tod2map requests over a pool of TODs.  Each result must be the same alone and in the mix:
map2tod bit for bit (the same rounded arithmetic per sample), tod2map within the float tolerance
against the oracle (float atomics reorder the sums).  A tight HBM budget forces plan evictions."""

import random
import time

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


def pool(seed, n=10, ny=256, nx=512):
    rng = np.random.default_rng(seed)
    xps = {i: random_raster(rng, int(rng.integers(1, 6)), 32 * int(rng.integers(16, 96)), ny, nx, True,
                            speed=float(rng.uniform(0.3, 1.1))) for i in range(n)}
    tods = {i: rng.standard_normal(x.shape[1:]).astype(np.float32) for i, x in xps.items()}
    return rng, xps, tods


def run_mix(g, xps_np, tods_np, m, requests, budget, ny=256, nx=512, jitter=True):
    import torch
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    xg = {i: torch.from_numpy(x).cuda() for i, x in xps_np.items()}
    tg = {i: torch.from_numpy(t).cuda() for i, t in tods_np.items()}
    in_map = torch.from_numpy(m).cuda()
    out_map = torch.zeros(3 * lp.npix, device="cuda")
    torch.cuda.synchronize()
    srv = g.PointingServer(xg, in_map, out_map, lp, hbm_budget_bytes=budget)
    futs = []
    rnd = random.Random(7)
    for kind, i in requests:
        futs.append((kind, i, srv.submit(kind, i, tod=tg[i] if kind == "tod2map" else None)))
        if jitter and rnd.random() < 0.3:
            time.sleep(rnd.uniform(0.0, 0.002))
    srv.drain()
    results = [(kind, i, f.result(timeout=30)) for kind, i, f in futs]
    srv.check()
    stats = srv.stats()
    srv.close()
    m2t = [(i, r.cpu().numpy()) for kind, i, r in results if kind == "map2tod"]
    return m2t, out_map.cpu().numpy(), stats, srv


def test_serving_mix_matches_alone(g):
    ny, nx = 256, 512
    rng, xps, tods = pool(3)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = rng.standard_normal(3 * lp_o.npix).astype(np.float32)
    kinds = ["plan"] * 4 + ["map2tod"] * 3 + ["tod2map"] * 3
    requests = [(kinds[int(rng.integers(0, 10))], int(rng.integers(0, len(xps)))) for _ in range(60)]
    m2t_mix, out_mix, stats, srv = run_mix(g, xps, tods, m, requests, budget=8 << 30)
    assert stats["launches"] >= 1 and not srv.errors
    # Alone: the same requests one at a time through the plain planned operators.
    import torch
    lpg = g.LocalPixelization.make_rectangle(ny, nx, True)
    lmap = g.LocalMap(lpg, torch.from_numpy(m).cuda())
    for i, r in m2t_mix:
        xg = torch.from_numpy(xps[i]).cuda()
        alone = torch.zeros(xps[i].shape[1:], device="cuda")
        g.map2tod(alone, lmap, xg, g.PointingPlan(g.PointingPrePlan(xg, ny, nx), xg))
        np.testing.assert_array_equal(r, alone.cpu().numpy())
    want = np.zeros(3 * lp_o.npix, np.float32)
    for kind, i in requests:
        if kind == "tod2map":
            oracle.tod2map(want, tods[i], xps[i], lp_o)
    rl1, mx = rel_stats(out_mix, want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_serving_tight_budget_evicts_and_stays_correct(g):
    ny, nx = 256, 512
    rng, xps, tods = pool(5, n=12)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = rng.standard_normal(3 * lp_o.npix).astype(np.float32)
    # Room for about three cached plans and six requests (the server's own accounting), not for all
    # twelve plans: plans are evicted and rebuilt as requests come and go.
    n_max = max(x[0].size for x in xps.values())
    per_plan = 16 * (n_max // 32) + (1 << 17) + (1 << 20)
    per_req = 4 * n_max + 16 * (n_max // 32) + (1 << 18)
    budget = 3 * per_plan + 6 * per_req
    requests = [("map2tod", i % 12) for i in range(36)] + [("tod2map", (5 * i) % 12) for i in range(24)]
    m2t_mix, out_mix, stats, srv = run_mix(g, xps, tods, m, requests, budget=budget, jitter=False)
    assert stats["evictions"] > 0 and stats["plan_cache"]["plans"] < 12, stats
    assert stats["plan_cache"]["bytes"] <= budget, stats
    import torch
    lpg = g.LocalPixelization.make_rectangle(ny, nx, True)
    lmap = g.LocalMap(lpg, torch.from_numpy(m).cuda())
    for i, r in m2t_mix:
        xg = torch.from_numpy(xps[i]).cuda()
        alone = torch.zeros(xps[i].shape[1:], device="cuda")
        g.map2tod(alone, lmap, xg, None)
        np.testing.assert_array_equal(r, alone.cpu().numpy())
    want = np.zeros(3 * lp_o.npix, np.float32)
    for kind, i in requests:
        if kind == "tod2map":
            oracle.tod2map(want, tods[i], xps[i], lp_o)
    rl1, mx = rel_stats(out_mix, want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_serving_rejects_bad_requests(g):
    import torch
    rng, xps, tods = pool(9, n=2)
    lp = g.LocalPixelization.make_rectangle(256, 512, True)
    xg = {i: torch.from_numpy(x).cuda() for i, x in xps.items()}
    srv = g.PointingServer(xg, torch.zeros(3 * lp.npix, device="cuda"), torch.zeros(3 * lp.npix, device="cuda"),
                           lp, hbm_budget_bytes=1 << 30)
    with pytest.raises(KeyError):
        srv.submit("map2tod", 99)
    with pytest.raises(ValueError):
        srv.submit("tod2map", 0)
    with pytest.raises(ValueError):
        srv.submit("bogus", 0)
    srv.close()


def test_serving_reports_errors_and_keeps_serving(g):
    """Device error bits of a launch fail that launch's requests and reach check(), which clears them;
    a request with bad arguments raises in submit(); the server goes on serving later requests."""
    import torch
    ny, nx = 256, 512
    rng, xps, tods = pool(13, n=3)
    xps[0] = xps[0].copy()
    xps[0][0, 0, 7] = ny + 3.0                       # a y outside the map in TOD 0
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    xg = {i: torch.from_numpy(x).cuda() for i, x in xps.items()}
    m = torch.from_numpy(rng.standard_normal(3 * lp.npix).astype(np.float32)).cuda()
    srv = g.PointingServer(xg, m, torch.zeros(3 * lp.npix, device="cuda"), lp, hbm_budget_bytes=1 << 30)
    try:
        with pytest.raises(RuntimeError, match="device error bits 0x1"):
            srv.submit("plan", 0).result(timeout=30)
        with pytest.raises(RuntimeError, match="device error bits"):
            srv.check()
        srv.check()                                       # cleared by the previous check()
        with pytest.raises(ValueError, match="shape"):
            srv.submit("tod2map", 1, tod=torch.zeros(7, device="cuda"))
        with pytest.raises(ValueError, match="float32"):
            srv.submit("tod2map", 1, tod=torch.zeros(xps[1].shape[1:], dtype=torch.float64, device="cuda"))
        futs = [srv.submit("map2tod", 1)] + [srv.submit("tod2map", 2, tod=torch.from_numpy(tods[2]).cuda())
                                             for _ in range(3)]
        r = futs[0].result(timeout=30)
        for f in futs[1:]:
            assert f.result(timeout=30) is None
        srv.check()
    finally:
        srv.close()
    alone = torch.zeros(xps[1].shape[1:], device="cuda")
    g.map2tod(alone, g.LocalMap(lp, m), xg[1], None)
    assert torch.equal(r, alone)
    g.serving.release_scratch()          # no server running: the shared scratch can go
    assert not g.serving._SCRATCH


def test_serving_waits_for_the_callers_stream(g):
    """Inputs written asynchronously on the caller's stream just before submit(): a TOD and the
    resident input map are filled by copies queued behind a long-running kernel on a side stream, and
    the requests are submitted from that stream without synchronising.  The server orders its launches
    after the caller's work, so tod2map and map2tod see the final inputs."""
    import torch
    ny, nx = 256, 512
    rng, xps, tods = pool(21, n=4)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    xg = {i: torch.from_numpy(x).cuda() for i, x in xps.items()}
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    m_src = torch.from_numpy(m).cuda()
    t_src = torch.from_numpy(tods[1]).cuda()
    in_map = torch.zeros(3 * lp.npix, device="cuda")
    out_map = torch.zeros(3 * lp.npix, device="cuda")
    tod = torch.zeros(xps[1].shape[1:], device="cuda")
    torch.cuda.synchronize()
    srv = g.PointingServer(xg, in_map, out_map, lp, hbm_budget_bytes=1 << 30)
    side = torch.cuda.Stream()
    try:
        with torch.cuda.stream(side):
            torch.cuda._sleep(50_000_000)                 # about 25 ms of GPU time on this stream
            tod.copy_(t_src)
            in_map.copy_(m_src)
            f_t2m = srv.submit("tod2map", 1, tod=tod)
            f_m2t = srv.submit("map2tod", 2)
        f_t2m.result(timeout=30)
        r = f_m2t.result(timeout=30)
        srv.check()
    finally:
        srv.close()
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, tods[1], xps[1], lp_o)
    rl1, mx = rel_stats(out_map.cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)
    want_t = np.zeros(xps[2].shape[1:], np.float32)
    oracle.map2tod(want_t, m, xps[2], lp_o)
    rl1, mx = rel_stats(r.cpu().numpy(), want_t)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)


def test_serving_idle_fast_path_and_batching(g):
    """A request submitted to an idle server is launched by submit() itself (no wait for the worker);
    a burst submitted at once is batched by the worker (fewer launches than requests); every map2tod
    result equals the plain planned operator's."""
    import torch
    ny, nx = 256, 512
    rng, xps, tods = pool(31, n=6)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    xg = {i: torch.from_numpy(x).cuda() for i, x in xps.items()}
    m = torch.from_numpy(rng.standard_normal(3 * lp.npix).astype(np.float32)).cuda()
    srv = g.PointingServer(xg, m, torch.zeros(3 * lp.npix, device="cuda"), lp, hbm_budget_bytes=1 << 30)
    try:
        r0 = srv.submit("map2tod", 0).result(timeout=30)
        assert srv.direct_launches == 1
        srv.drain()
        futs = [(i % 6, srv.submit("map2tod", i % 6)) for i in range(24)]
        outs = [(i, f.result(timeout=30)) for i, f in futs]
        assert srv.launches < 1 + 24
        srv.check()
    finally:
        srv.close()
    lmap = g.LocalMap(lp, m)
    for i, r in [(0, r0)] + outs:
        alone = torch.empty(xps[i].shape[1:], device="cuda")
        g.map2tod(alone, lmap, xg[i], g.PointingPlan(g.PointingPrePlan(xg[i], ny, nx), xg[i]))
        assert torch.equal(r, alone)
