"""Shared helpers for the tests (not a test module)."""

import numpy as np


def literal_enumerate(iy0, iy1, ix0, ix1):
    """cell_enumerator::enumerate written out literally (gpu_mm_internals.hpp:194-221): the six
    (iycell, ixcell) slot pairs ca0..ca5 of PointingPlan.cu:173-178."""
    def process_pair(c0, c1):
        c1 = c1 if c0 != c1 else -1
        flag = c0 & 1
        even = c1 if flag else c0
        odd = c0 if flag else c1
        return even, odd

    y0, y1 = process_pair(iy0 >> 6, iy1 >> 6)
    x0, x1 = process_pair(ix0 >> 6, ix1 >> 6)
    x2 = -1 if (x0 != 0 and x1 != 0) else 0
    x0 = x0 if x0 != 0 else -1
    x1 = x1 if x1 != 0 else -1
    return [(y0, x0), (y0, x1), (y0, x2), (y1, x0), (y1, x1), (y1, x2)]


def literal_plan_words(located, nsamp):
    """Simulates the reference's plan_kernel (PointingPlan.cu:121-231 with W=4) warp by warp:
    cell_analysis (match_any + ballot over the 32 lanes, each cell at its highest lane),
    mt_ringbuf::absorb with its running
    nmt_local / na_cumul, and the per-line na_cumul reset.  'located' is a list of
    (iy0, iy1, ix0, ix1) per sample.  Returns the emitted 64-bit words (unordered)."""
    ncl = nsamp // 32
    c = max(16, (ncl + 1023) // 1024)
    c = (c + 3) & ~3
    nblocks = (ncl + c - 1) // c
    words = []
    for b in range(nblocks):
        l0, l1 = b * c, min(ncl, (b + 1) * c)
        for w in range(4):
            nmt_local = 0
            for cl in range(l0 + w, l1, 4):
                slots = [literal_enumerate(*located[32 * cl + lane]) for lane in range(32)]
                cas = []
                for k in range(6):
                    icells = [(((iy << 10) | ix) & 0xFFFFFFFF, (iy >= 0) and (ix >= 0)) for (iy, ix) in
                              (slots[lane][k] for lane in range(32))]
                    active = []
                    for lane in range(32):
                        v, valid = icells[lane]
                        # cell_analysis (PointingPlan.cu:27-35): is_lowest = ((mmask >> lane) == 1),
                        # which holds at the HIGHEST lane of the matching lanes.
                        highest = all(icells[j][0] != v for j in range(lane + 1, 32))
                        if valid and highest:
                            active.append(v)
                    cas.append(active)
                mflag = sum(len(a) for a in cas) > 1
                na_cumul = 0
                for active in cas:
                    na = len(active)
                    if na == 0:
                        continue
                    for j, v in enumerate(active):
                        zflag = mflag and (na_cumul == 0) and (j == 0)
                        words.append(v | (cl << 20) | (int(mflag) << 46) | (int(zflag) << 47))
                    nmt_local += na
                    if nmt_local >= 32:
                        nmt_local -= 32
                        na_cumul += na
    return words


def canonical(words):
    """Sort mt words by (cell, cache line)."""
    w = np.asarray(words, dtype=np.uint64)
    key = (w & np.uint64(0xFFFFF)) * np.uint64(1 << 26) + ((w >> np.uint64(20)) & np.uint64((1 << 26) - 1))
    return w[np.argsort(key, kind="stable")]


def rel_stats(a, b):
    """(rel-L1 as in the reference's tests.py:220-224, max |a-b| / max |b|)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = np.abs(a).sum() + np.abs(b).sum()
    rl1 = float(np.abs(a - b).sum() / den) if den > 0 else 0.0
    mx = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)) if a.size else 0.0
    return rl1, mx


def random_raster(rng, ndet, nt, ny, nx, periodic, speed=0.7, ydrift=0.01, yspread=3.0):
    """Small raster scans (float32 (3, ndet, nt)) with random phases; x crosses the wrap if periodic."""
    t = np.arange(nt, dtype=np.float64)
    xp = np.zeros((3, ndet, nt))
    L = nx - 1.0
    for d in range(ndet):
        x = np.abs(np.remainder(speed * t + rng.uniform(0, 2 * L), 2 * L) - L)
        if periodic:
            x = np.remainder(x + rng.uniform(0, nx), nx)
        else:
            x = np.clip(x, 0, nx - 2.001)
        y = rng.uniform(1, max(1.5, ny - 2 - ydrift * nt - yspread * 4)) + ydrift * t + yspread * (d % 4)
        xp[0, d] = np.clip(y, 0, ny - 1.0)
        xp[1, d] = x
        xp[2, d] = rng.uniform(0, 2 * np.pi) + 2 * np.pi * t / 700.0
    return xp.astype(np.float32)
