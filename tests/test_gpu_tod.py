"""GPU tests of the TOD preprocessing kernels (deglitching, cut ranges, clip) against the CPU
restatements of the reference's Python reference implementations (gpu_mm.py:1504-1563) and of its
kernels' loops (cuts.cu:16-36, misc.cu:8-19)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import gpu_mm_b200
    return gpu_mm_b200


def cuda(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def cut_tables(rng, ndet, nt, per_det=5):
    """Sorted, disjoint cut ranges per detector (some empty detectors), as the deglitching index maps."""
    ranges, dets = [], []
    for d in range(ndet):
        k = int(rng.integers(0, per_det + 1))
        ts = np.sort(rng.choice(np.arange(8, nt - 8), size=2 * k, replace=False))
        for j in range(k):
            ranges.append((ts[2 * j], ts[2 * j + 1]))
            dets.append(d)
    R = len(ranges)
    im = np.zeros((R, 5), np.int32)
    im2 = np.zeros((R, 4), np.int32)
    first = {}
    for r, (d, (t1, t2)) in enumerate(zip(dets, ranges)):
        first.setdefault(d, r)
        im[r] = (d, max(0, t1 - 6), t1, t2, min(nt, t2 + 6))
        im2[r] = (d, first[d], t1, t2)
    im[0, 1:3] = im[0, 2]          # one empty border range
    return im, im2


def test_border_means_and_deglitch(g):
    rng = np.random.default_rng(0)
    ndet, nt = 12, 3000
    sig = rng.standard_normal((ndet, nt)).astype(np.float32) + np.repeat(rng.uniform(-5, 5, (ndet, 1)), nt, 1).astype(np.float32)
    im, im2 = cut_tables(rng, ndet, nt)
    R = len(im)
    out = cuda(np.zeros((R, 2), np.float32))
    g.get_border_means(out, cuda(sig), cuda(im))
    want = g.reference_get_border_means(sig, im)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-5, atol=1e-6)
    s_gpu = cuda(sig)
    g.deglitch(s_gpu, cuda(want), cuda(im2))
    s_ref = sig.copy()
    g.reference_deglitch(s_ref, want, im2)
    np.testing.assert_allclose(s_gpu.cpu().numpy(), s_ref, rtol=1e-5, atol=1e-4)


def test_ranges_and_clip(g):
    import torch
    rng = np.random.default_rng(1)
    ndet, nsamp = 7, 500
    tod = rng.standard_normal((ndet, nsamp)).astype(np.float32)
    nr = 20
    dets = rng.integers(0, ndet, nr).astype(np.int32)
    starts = rng.integers(0, nsamp - 40, nr).astype(np.int32)
    lens = rng.integers(0, 40, nr).astype(np.int32)
    offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int32)
    junk = cuda(np.zeros(int(lens.sum()), np.float32))
    t = cuda(tod)
    g.extract_ranges(t, junk, cuda(offs), cuda(dets), cuda(starts), cuda(lens))
    want = np.concatenate([tod[d, s:s + n] for d, s, n in zip(dets, starts, lens)])
    np.testing.assert_array_equal(junk.cpu().numpy(), want)
    g.clear_ranges(t, cuda(dets), cuda(starts), cuda(lens))
    cleared = tod.copy()
    for d, s, n in zip(dets, starts, lens):
        cleared[d, s:s + n] = 0
    np.testing.assert_array_equal(t.cpu().numpy(), cleared)
    g.insert_ranges(t, junk, cuda(offs), cuda(dets), cuda(starts), cuda(lens))
    restored = cleared.copy()
    jn = junk.cpu().numpy()
    for d, s, n, o in zip(dets, starts, lens, offs):
        restored[d, s:s + n] = jn[o:o + n]
    np.testing.assert_array_equal(t.cpu().numpy(), restored)
    c = cuda(tod)
    g.clip(c, -0.5, 0.75)
    np.testing.assert_array_equal(c.cpu().numpy(), np.maximum(-0.5, np.minimum(0.75, tod)))
    # Index maps out of range are refused (nothing is written outside the arrays).
    bad = starts.copy()
    bad[3] = nsamp
    lens2 = lens.copy()
    lens2[3] = 5
    with pytest.raises(RuntimeError):
        g.clear_ranges(t, cuda(dets), cuda(bad), cuda(lens2))
    with pytest.raises(RuntimeError):
        out = cuda(np.zeros((1, 2), np.float32))
        g.get_border_means(out, cuda(tod), cuda(np.array([[ndet, 0, 5, 5, 9]], np.int32)))
