"""CPU tests of the oracle: pinned against the reference's own code (golden vectors produced by
oracle/_ref from the reference header, plus a live comparison when oracle/_ref is built here) and
against literal restatements of the reference's plan construction."""

import numpy as np
import pytest

import oracle
from tests._common import canonical, literal_enumerate, literal_plan_words, random_raster

CASES = ("wrap_rect", "flat_cells_accum", "partial_missing", "scattered", "errors")


def _lpix(golden, name):
    p = golden[f"{name}__params"]
    ny, nx, periodic, ys, ps = int(p[0]), int(p[1]), bool(p[2]), int(p[3]), int(p[4])
    return oracle.Lpix(ny, nx, golden[f"{name}__cell_offsets"], ys, ps, periodic), p


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden_ops(golden_ops, name):
    """The C restatement reproduces the reference header's map2tod/tod2map bit for bit."""
    lp, p = _lpix(golden_ops, name)
    partial, accum = bool(p[5]), bool(p[6])
    xp = golden_ops[f"{name}__xpointing"]
    m = golden_ops[f"{name}__map"].astype(np.float32)
    tod = golden_ops[f"{name}__tod_init"].astype(np.float32)
    e1 = oracle.map2tod(tod, m, xp, lp, partial, accum)
    assert e1 == int(p[7])
    np.testing.assert_array_equal(tod, golden_ops[f"{name}__m2t_out"])
    mo = np.zeros(3 * lp.npix, dtype=np.float32)
    e2 = oracle.tod2map(mo, golden_ops[f"{name}__tod_in"].astype(np.float32), xp, lp, partial)
    assert e2 == int(p[8])
    np.testing.assert_array_equal(mo, golden_ops[f"{name}__t2m_out"])


@pytest.mark.parametrize("name", CASES[:4])
def test_plan_oracle_matches_golden_tester(golden_ops, golden_plans, name):
    """nmt_cumsum and the sorted 46-bit mt multiset equal PointingPlanTester's (tests.py:227-254),
    and mflag marks exactly the lines touching more than one cell."""
    p = golden_ops[f"{name}__params"]
    ny, nx, periodic = int(p[0]), int(p[1]), bool(p[2])
    xp = golden_ops[f"{name}__xpointing"]
    pp = oracle.preplan(xp, ny, nx, periodic)
    cum = golden_plans[f"{name}__nmt_cumsum"]
    np.testing.assert_array_equal(pp["nmt_cumsum"][:len(cum)], cum)
    assert np.all(pp["nmt_cumsum"][len(cum):] == cum[-1])
    mt, owner, err = oracle.plan(xp, ny, nx, periodic)
    assert err == 0
    np.testing.assert_array_equal(np.sort(mt & np.uint64((1 << 46) - 1)), golden_plans[f"{name}__sorted46"])
    counts = golden_plans[f"{name}__line_counts"]
    cl = ((mt >> np.uint64(20)) & np.uint64((1 << 26) - 1)).astype(np.int64)
    mflag = ((mt >> np.uint64(46)) & np.uint64(1)).astype(bool)
    np.testing.assert_array_equal(mflag, counts[cl] > 1)


def _locate_all(xp, ny, nx, periodic):
    xpf = xp.reshape(3, -1)
    out = []
    for s in range(xpf.shape[1]):
        (iy0, iy1, ix0, ix1), _, _ = oracle.locate(xpf[0, s], xpf[1, s], ny, nx, periodic)
        out.append((iy0, iy1, ix0, ix1))
    return out


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_plan_oracle_matches_literal_ring_buffer(seed):
    """Full 64-bit plan words (mflag, zflag included) equal a literal simulation of the reference's
    per-warp ring buffer, in canonical (cell, cache line) order."""
    rng = np.random.default_rng(seed)
    ny, nx = 150, 260
    if seed == 2:
        # Scattered pointing: up to ~100 cells per line, so ring-buffer flushes happen mid-line.
        n = 32 * 96
        xp = np.zeros((3, n), dtype=np.float32)
        xp[0] = rng.uniform(0, ny - 1, n)
        xp[1] = rng.uniform(0, nx, n)
        xp[2] = 1.0
    else:
        xp = random_raster(rng, 6, 1024 + 32 * seed, ny, nx, periodic=True, speed=0.9 + 2.0 * seed)
    mt, owner, err = oracle.plan(xp, ny, nx, True)
    assert err == 0
    sim = canonical(literal_plan_words(_locate_all(xp, ny, nx, True), xp.size // 3))
    np.testing.assert_array_equal(mt, sim)
    # Canonical order and per-line flag invariants (map2tod.cu:18-43 needs >= 1 zflag per mflag line).
    key = (mt & np.uint64(0xFFFFF)) * np.uint64(1 << 26) + ((mt >> np.uint64(20)) & np.uint64((1 << 26) - 1))
    assert np.all(np.diff(key.astype(np.float64)) > 0)
    cl = ((mt >> np.uint64(20)) & np.uint64((1 << 26) - 1)).astype(np.int64)
    z = ((mt >> np.uint64(47)) & np.uint64(1)).astype(np.int64)
    mf = ((mt >> np.uint64(46)) & np.uint64(1)).astype(bool)
    zc = np.bincount(cl, weights=z, minlength=xp.size // 96)
    mline = np.zeros(xp.size // 96, dtype=bool)
    mline[cl[mf]] = True
    assert np.all(zc[mline] >= 1)
    assert np.all(zc[~mline] == 0)


def test_owner_bits_mark_lowest_cell_per_line():
    rng = np.random.default_rng(5)
    xp = random_raster(rng, 4, 2048, 200, 300, periodic=True, speed=0.8)
    mt, owner, err = oracle.plan(xp, 200, 300, True)
    bits = np.unpackbits(owner.view(np.uint8), bitorder="little")[:len(mt)].astype(bool)
    cl = ((mt >> np.uint64(20)) & np.uint64((1 << 26) - 1)).astype(np.int64)
    cell = (mt & np.uint64(0xFFFFF)).astype(np.int64)
    ncl = xp.size // 96
    assert np.bincount(cl[bits], minlength=ncl).tolist() == [1] * ncl
    mins = np.full(ncl, 1 << 30)
    np.minimum.at(mins, cl, cell)
    np.testing.assert_array_equal(cell[bits], mins[cl[bits]])


def test_slots_match_literal_enumerate():
    rng = np.random.default_rng(7)
    ny, nx = 300, 400
    n = 4096
    xp = np.zeros((3, n), dtype=np.float32)
    xp[0] = rng.uniform(0, ny - 1, n)
    xp[1] = rng.uniform(-nx, 2 * nx, n)
    # Exact cell boundaries and the wrap point.
    xp[1, :64] = np.arange(64) * 64.0 - 1.0
    xp[1, 64:70] = [nx - 1, nx, -nx, 2 * nx, 0.0, nx - 0.5]
    slots = oracle.sample_slots(xp, ny, nx, True)
    for s, (iy0, iy1, ix0, ix1) in enumerate(_locate_all(xp, ny, nx, True)):
        lit = [((a << 10) | b) if (a >= 0 and b >= 0) else -1 for (a, b) in literal_enumerate(iy0, iy1, ix0, ix1)]
        assert slots[s].tolist() == lit, s


def test_locate_matches_reference_header():
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source tree)")
    rng = np.random.default_rng(11)
    for (ny, nx, periodic) in ((100, 200, True), (100, 200, False), (64, 64, True), (2, 2, True)):
        ys = np.concatenate([rng.uniform(-3, ny + 3, 300), [0, ny - 1, ny - 2, 0.5, ny - 1.0001]])
        xs = np.concatenate([rng.uniform(-2 * nx, 3 * nx, 300), [0, nx - 1, nx, -nx, 2 * nx, -nx - 0.5, 2 * nx + 0.5]])
        for y in ys.astype(np.float32):
            for x in xs[::7].astype(np.float32):
                a = oracle.locate(y, x, ny, nx, periodic)
                b = oracle.locate(y, x, ny, nx, periodic, use_ref=True)
                assert a[2] == b[2]
                if a[2] == 0:
                    assert a[0] == b[0] and a[1] == b[1], (y, x)


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_matches_reference_header_live(seed):
    """Random cases against oracle/_ref (the reference's own header), bit for bit, float32 and float64."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference source tree)")
    rng = np.random.default_rng(100 + seed)
    ny, nx = 140, 330
    periodic = bool(seed)
    xp = random_raster(rng, 8, 512, ny, nx, periodic)
    lp = oracle.Lpix.rectangle(ny, nx, periodic)
    for dt in (np.float32, np.float64):
        m = rng.standard_normal(3 * lp.npix).astype(dt)
        x = xp.astype(dt)
        t1 = rng.standard_normal(xp.shape[1:]).astype(dt)
        t2 = t1.copy()
        assert oracle.map2tod(t1, m, x, lp, False, True) == oracle.map2tod(t2, m, x, lp, False, True, use_ref=True)
        np.testing.assert_array_equal(t1, t2)
        m1 = np.zeros_like(m)
        m2 = np.zeros_like(m)
        oracle.tod2map(m1, t1, x, lp)
        oracle.tod2map(m2, t1, x, lp, use_ref=True)
        np.testing.assert_array_equal(m1, m2)


def test_preplan_geometry():
    """ncl_per_threadblock, planner_nblocks, nmt_per_threadblock, pointing_nblocks follow
    PointingPrePlan.cu:162-165 and :236-238."""
    rng = np.random.default_rng(3)
    xp = random_raster(rng, 2, 32 * 700, 100, 100, True)
    pp = oracle.preplan(xp, 100, 100, True)
    ncl = xp.size // 96
    c = max(16, -(-ncl // 1024))
    c = (c + 3) & ~3
    assert pp["ncl_per_threadblock"] == c
    assert pp["planner_nblocks"] == -(-ncl // c)
    npt = (int(np.sqrt(pp["nmt"])) + 32) & ~31
    assert pp["nmt_per_threadblock"] == npt
    assert pp["pointing_nblocks"] == -(-pp["nmt"] // npt)


def test_errors_reported():
    rng = np.random.default_rng(9)
    xp = random_raster(rng, 2, 64, 50, 80, False)
    lp = oracle.Lpix.rectangle(50, 80, False)
    m = np.zeros(3 * lp.npix, np.float32)
    t = np.zeros(xp.shape[1:], np.float32)
    assert oracle.map2tod(t, m, xp, lp) == 0
    xp[0, 0, 3] = 49.5
    assert oracle.map2tod(t, m, xp, lp) == oracle.ERR_BAD_YPIX
    xp[0, 0, 3] = 10.0
    xp[1, 1, 5] = 78.5
    assert oracle.map2tod(t, m, xp, lp) == oracle.ERR_BAD_XPIX
    xp[1, 1, 5] = 10.0
    offs = lp.cell_offsets.copy()
    offs[0, 0] = -1
    lp2 = oracle.Lpix(50, 80, offs, lp.ystride, lp.polstride, False)
    assert oracle.map2tod(t, m, xp, lp2) & oracle.ERR_NOT_IN_PIXELIZATION


@pytest.mark.parametrize("ny,nx,periodic", [(300, 400, True), (300, 400, False), (130, 64, True), (200, 128, True),
                                            (65536, 65536, True)])
def test_line_count_is_distinct_cells(ny, nx, periodic):
    """A cache line's number of (cell, line) pairs -- distinct valid (slot, cell) values over its 32
    samples' six cell_enumerator slots -- equals its number of distinct cells among the samples'
    bilinear neighbours: each cell's slot is fixed by its own coordinates (row parity; column 0 or
    column parity).  The preplan's warp-reduction count relies on this.  Lines: scans near cell
    corners, the x wrap, and scattered samples."""
    rng = np.random.default_rng(ny + nx + periodic)
    nl = 96
    xp = np.zeros((3, nl, 32), dtype=np.float64)
    t = np.arange(32)
    for i in range(nl):
        kind = i % 3
        y0 = rng.uniform(0, ny - 2)
        x0 = rng.uniform(-nx if periodic else 0, (2 * nx if periodic else nx - 1))
        if kind == 0:       # a scan through a cell corner
            cy, cx = 64 * rng.integers(1, max(2, ny // 64)), 64 * rng.integers(0, max(1, nx // 64))
            y0, x0 = cy - rng.uniform(0, 1.5), cx - rng.uniform(0, 20)
        if kind == 2:       # scattered samples
            xp[0, i] = rng.uniform(0, ny - 1, 32)
            xp[1, i] = rng.uniform(-nx if periodic else 0, (2 * nx if periodic else nx - 1), 32)
            continue
        sp = rng.choice([-1.0, 1.0]) * rng.uniform(0.2, 1.2)
        xp[0, i] = np.clip(y0 + 0.01 * t, 0, ny - 1)
        x = x0 + sp * t
        xp[1, i] = x if periodic else np.clip(x, 0, nx - 1)
    xp = xp.astype(np.float32)
    counts = oracle.line_counts(xp, ny, nx, periodic)
    located = _locate_all(xp, ny, nx, periodic)
    for line in range(nl):
        cells = set()
        for (iy0, iy1, ix0, ix1) in located[32 * line: 32 * line + 32]:
            for iy in (iy0, iy1):
                for ix in (ix0, ix1):
                    cells.add((iy >> 6, ix >> 6))
        assert counts[line] == len(cells), (line, counts[line], sorted(cells))
