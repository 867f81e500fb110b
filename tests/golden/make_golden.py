"""Generates the golden vectors in tests/golden/ (committed; run once where the reference tree exists).

  python tests/golden/make_golden.py

Operator outputs come from oracle/_ref, i.e. the reference's own include/gpu_mm_internals.hpp
templates (pixel_locator, map_evaluator, map_accumulator) driven by the sample loops of
map2tod_reference.cu / tod2map_reference.cu.  Plan vectors (nmt_cumsum, sorted mt multiset, per-line
cell counts) come from a direct numpy restatement of PointingPlanTester.cu:126-160 fed with the
reference header's own locate() output -- an independent route from oracle.c's slot machinery.

Inputs are stored with the outputs, so the tests never regenerate them.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def rect_cells(ny, nx):
    nyc, nxc = (ny + 63) // 64, (nx + 63) // 64
    offs = 64 * np.arange(nxc)[None, :] + 64 * 64 * nxc * np.arange(nyc)[:, None]
    return offs.astype(np.int64), 64 * nxc, 64 * 64 * nyc * nxc


def cellmajor(ny, nx, present):
    """Cell-major layout (ystride=64, polstride=4096) for the cells where present[iyc, ixc]."""
    offs = np.full(present.shape, -1, dtype=np.int64)
    k = 0
    for iy in range(present.shape[0]):
        for ix in range(present.shape[1]):
            if present[iy, ix]:
                offs[iy, ix] = 3 * 64 * 64 * k
                k += 1
    return offs, 64, 64 * 64


def raster(rng, ndet, nt, ny, nx, speed, periodic, y0, ydrift):
    t = np.arange(nt, dtype=np.float64)
    xp = np.zeros((3, ndet, nt))
    L = nx - 1.0
    for d in range(ndet):
        x = np.abs(np.remainder(speed * t + rng.uniform(0, 2 * L), 2 * L) - L) + 3 * (d % 4)
        if periodic:
            x = np.remainder(x + rng.uniform(-5, 5), nx)
        else:
            x = np.clip(x, 0, nx - 2.001)
        xp[0, d] = np.clip(y0 + ydrift * t + 3 * (d // 4), 0, ny - 1)
        xp[1, d] = x
        xp[2, d] = 2 * np.pi * np.remainder(t / 512.0 + d / ndet, 1.0)
    return xp.astype(np.float32)


def tester_plan(xp, ny, nx, periodic):
    """PointingPlanTester.cu:126-160 with (iy0, ix0) from the reference header's locate()."""
    xpf = xp.reshape(3, -1)
    nsamp = xpf.shape[1]
    iy = np.zeros(nsamp, dtype=np.int64)
    ix = np.zeros(nsamp, dtype=np.int64)
    for s in range(nsamp):
        (iy0, _, ix0, _), _, _ = oracle.locate(xpf[0, s], xpf[1, s], ny, nx, periodic, use_ref=True)
        iy[s], ix[s] = iy0, ix0
    ncl = nsamp // 32
    c = max(16, (ncl + 1023) // 1024)
    c = (c + 3) & ~3
    nblocks = (ncl + c - 1) // c
    cum = np.zeros(nblocks, dtype=np.uint32)
    words, counts = [], np.zeros(ncl, dtype=np.int64)
    n = 0
    for b in range(nblocks):
        for cl in range(b * c, min(ncl, (b + 1) * c)):
            cells = set()
            for s in range(32 * cl, 32 * cl + 32):
                ix1 = ix[s] + 1 if ix[s] < nx - 1 else 0
                for (yy, xx) in ((iy[s], ix[s]), (iy[s], ix1), (iy[s] + 1, ix[s]), (iy[s] + 1, ix1)):
                    cells.add(((yy >> 6) << 10) | (xx >> 6))
            counts[cl] = len(cells)
            words += [cc | (cl << 20) for cc in cells]
            n += len(cells)
        cum[b] = n
    return cum, np.sort(np.array(words, dtype=np.uint64)), counts


def op_case(name, rng, ndet, nt, ny, nx, periodic, layout, partial, accum, speed=0.7, y0=5.0, ydrift=0.01,
            xp=None, missing=None):
    if xp is None:
        xp = raster(rng, ndet, nt, ny, nx, speed, periodic, y0, ydrift)
    if layout == "rect":
        offs, ys, ps = rect_cells(ny, nx)
    else:
        nyc, nxc = (ny + 63) // 64, (nx + 63) // 64
        present = np.ones((nyc, nxc), dtype=bool)
        if missing is not None:
            for (a, b) in missing:
                present[a, b] = False
        offs, ys, ps = cellmajor(ny, nx, present)
    lp = oracle.Lpix(ny, nx, offs, ys, ps, periodic)
    # Map and TOD inputs are N(0,1) rounded to float16 (stored as float16, exact in float32) to keep
    # the fixture small; the tod2map output starts from a zero map.
    m = rng.standard_normal(3 * lp.npix).astype(np.float16)
    tod_in = rng.standard_normal(xp.shape[1:]).astype(np.float16)
    tod_init = (rng.standard_normal(xp.shape[1:]) if accum else np.zeros(xp.shape[1:])).astype(np.float16)
    tod_out = tod_init.astype(np.float32)
    e1 = oracle.map2tod(tod_out, m.astype(np.float32), xp, lp, partial, accum, use_ref=True)
    m_out = np.zeros(3 * lp.npix, dtype=np.float32)
    e2 = oracle.tod2map(m_out, tod_in.astype(np.float32), xp, lp, partial, use_ref=True)
    return {f"{name}__xpointing": xp, f"{name}__cell_offsets": offs, f"{name}__map": m, f"{name}__tod_in": tod_in,
            f"{name}__tod_init": tod_init, f"{name}__m2t_out": tod_out, f"{name}__t2m_out": m_out,
            f"{name}__params": np.array([ny, nx, int(periodic), ys, ps, int(partial), int(accum), e1, e2],
                                        dtype=np.int64)}


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built: run 'make -C oracle ref' where the reference tree exists")
    rng = np.random.default_rng(20261203)
    ops = {}
    # Periodic raster crossing the x wrap, rectangle layout, non-multiple-of-64 map.
    ops.update(op_case("wrap_rect", rng, 4, 512, 60, 150, True, "rect", False, False, speed=0.9, y0=2.0, ydrift=0.05))
    # Non-periodic, cell-major layout, accum=True.
    ops.update(op_case("flat_cells_accum", rng, 4, 512, 100, 130, False, "cells", False, True, y0=50.0))
    # Partial pixelization with missing cells.
    ops.update(op_case("partial_missing", rng, 4, 512, 100, 192, True, "cells", True, False, y0=50.0,
                       missing=[(0, 1), (1, 2)]))
    # Scattered pointing: every sample somewhere random (many cells per cache line), with x
    # values in the periodic fold range [-nx, 2nx].
    ny, nx = 70, 140
    xs = np.zeros((3, 1024), dtype=np.float32)
    xs[0] = rng.uniform(0, ny - 1, 1024)
    xs[1] = rng.uniform(-nx, 2 * nx, 1024)
    xs[2] = rng.uniform(0, 2 * np.pi, 1024)
    ops.update(op_case("scattered", rng, 0, 0, ny, nx, True, "rect", False, False, xp=xs))
    # Error case: y out of range -> bit 1, x out of range (non-periodic) -> bit 2.
    xe = raster(rng, 2, 256, 60, 100, 0.5, False, 3.0, 0.0)
    xe[0, 0, 7] = -2.0
    xe[1, 1, 9] = 500.0
    ops.update(op_case("errors", rng, 0, 0, 60, 100, False, "rect", False, False, xp=xe))
    np.savez_compressed(os.path.join(HERE, "golden_ops.npz"), **ops)

    plans = {}
    for name in ("wrap_rect", "flat_cells_accum", "partial_missing", "scattered"):
        p = ops[f"{name}__params"]
        xp = ops[f"{name}__xpointing"]
        cum, words, counts = tester_plan(xp, int(p[0]), int(p[1]), bool(p[2]))
        plans[f"{name}__nmt_cumsum"] = cum
        plans[f"{name}__sorted46"] = words
        plans[f"{name}__line_counts"] = counts
    np.savez_compressed(os.path.join(HERE, "golden_plans.npz"), **plans)
    for f in ("golden_ops.npz", "golden_plans.npz"):
        print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
