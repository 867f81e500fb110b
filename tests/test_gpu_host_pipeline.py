"""GPU tests of gpu_mm_b200.HostPipeline: planned map2tod / tod2map over TODs in pinned host memory,
streamed in chunks of detectors.  map2tod must equal the plain planned operator bit for bit (the
same per-sample arithmetic); tod2map must match the oracle within the float tolerance (float
atomics reorder the sums).  Chunks that do not divide the detectors, a detector count that is not a
multiple of 32 samples per detector, host and device maps, and two runs in a row are covered."""

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


def pinned(a):
    import torch
    t = torch.empty(a.shape, dtype=torch.float32, pin_memory=True)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)))
    return t


@pytest.mark.parametrize("ndet,nt,chunk_dets,host_maps", [(7, 1024, 2, False), (10, 1008, 3, True),
                                                          (5, 4096, None, True)])
def test_host_pipeline_matches_plain(g, ndet, nt, chunk_dets, host_maps):
    import torch
    ny, nx = 256, 512
    rng = np.random.default_rng(ndet * 1000 + nt)
    xp = random_raster(rng, ndet, nt, ny, nx, True)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    m = rng.standard_normal(3 * lp.npix).astype(np.float32)
    pipe = g.HostPipeline(lp, ndet, nt, chunk_dets=chunk_dets)
    assert len(pipe.chunks) >= 1 and all((d1 - d0) * nt % 32 == 0 for d0, d1 in pipe.chunks)

    # The plain planned operators on the whole TOD, for map2tod.
    xg = torch.from_numpy(xp).cuda()
    plan = g.PointingPlan(g.PointingPrePlan(xg, ny, nx), xg)
    want_tod = torch.zeros((ndet, nt), device="cuda")
    g.map2tod(want_tod, g.LocalMap(lp, torch.from_numpy(m).cuda()), xg, plan)
    want_tod = want_tod.cpu().numpy()

    xp_h = pinned(xp)
    for rep in range(2):
        tin = rng.standard_normal((ndet, nt)).astype(np.float32)
        tin_h = pinned(tin)
        tout_h = pinned(np.full((ndet, nt), np.nan, np.float32))
        m0 = rng.standard_normal(3 * lp.npix).astype(np.float32)   # tod2map accumulates into this
        if host_maps:
            min_ = pinned(m)
            mout = pinned(m0)
        else:
            min_ = g.LocalMap(lp, torch.from_numpy(m).cuda())
            mout = g.LocalMap(lp, torch.from_numpy(m0).cuda())
        pipe.run(xp_h, map_in=min_, tod_out=tout_h, tod_in=tin_h, map_out=mout)
        pipe.wait()
        np.testing.assert_array_equal(tout_h.numpy(), want_tod)
        got_map = mout.numpy() if host_maps else mout.arr.cpu().numpy()
        want_map = m0.copy()
        oracle.tod2map(want_map, tin, xp, lp_o)
        rl1, mx = rel_stats(got_map - m0, want_map - m0)
        assert rl1 < RL1_TOL and mx < MAX_TOL, (rep, rl1, mx)


def test_host_pipeline_tod2map_only_and_errors(g):
    import torch
    ny, nx = 128, 256
    rng = np.random.default_rng(11)
    ndet, nt = 4, 2048
    xp = random_raster(rng, ndet, nt, ny, nx, True)
    lp = g.LocalPixelization.make_rectangle(ny, nx, True)
    lp_o = oracle.Lpix.rectangle(ny, nx, True)
    pipe = g.HostPipeline(lp, ndet, nt, chunk_dets=1, nslots=2)
    tin = rng.standard_normal((ndet, nt)).astype(np.float32)
    out = torch.zeros(3 * lp.npix, device="cuda")
    pipe.run(pinned(xp), tod_in=pinned(tin), map_out=out)
    pipe.wait()
    want = np.zeros(3 * lp.npix, np.float32)
    oracle.tod2map(want, tin, xp, lp_o)
    rl1, mx = rel_stats(out.cpu().numpy(), want)
    assert rl1 < RL1_TOL and mx < MAX_TOL, (rl1, mx)

    # Pageable host memory and wrong shapes are rejected before anything is queued.
    with pytest.raises(RuntimeError, match="pinned"):
        pipe.run(torch.from_numpy(xp), tod_in=pinned(tin), map_out=out)
    with pytest.raises(RuntimeError, match="shape"):
        pipe.run(pinned(xp[:, :2]), tod_in=pinned(tin), map_out=out)
    with pytest.raises(RuntimeError, match="multiple of 32"):
        g.HostPipeline(lp, 3, 7)

    # A sample outside the map (non-periodic y) is reported after the run, like the plain operator.
    bad = xp.copy()
    bad[0, 2, 100] = ny + 5.0
    pipe.run(pinned(bad), tod_in=pinned(tin), map_out=out)
    with pytest.raises(RuntimeError):
        pipe.wait()
