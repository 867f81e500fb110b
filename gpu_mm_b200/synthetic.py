"""Seeded synthetic inputs for the pointing operators.

The reference measures on ACT xpointing files that are not available here; these raster scans stand
in for them, with the shapes, sizes and value ranges of the benchmark configurations:

* ``raster_xpointing``: a grid of detectors sweeping back and forth in x (triangle wave at a given
  speed in pixels per sample), drifting slowly in y, with detector angles
  ``alpha = 2*pi*frac(t/4096 + d/ndet)``.  Computed in float64, stored as float32.
* ``config1`` / ``config2`` / ``config3``: the small (2^22 samples, 3x1024x2048 map), large
  (2^28 samples, 3x8192x32768 map, hit cells only) and high-hit (2^28 samples in a 512x512 box)
  workloads.

Everything is generated with torch so that the large cases can be built directly on the GPU.
"""

import math

import numpy as np
import torch


def triangle(v, length):
    """Triangle wave starting at 0, rising to 'length' and back, period 2*length."""
    p = torch.remainder(v, 2.0 * length)
    return length - torch.abs(p - length)


def raster_xpointing(ndet_y, ndet_x, nt, spacing, speed, nxpix, y0, ydrift, xlo=0.0, xspan=None,
                     yspan=None, yspeed=None, alpha_period=4096.0, wrap_x=True, device="cpu", dtype=torch.float32):
    """Returns xpointing of shape (3, ndet_y*ndet_x, nt), rows (y, x, alpha).

    Detector d = ndet_x*i + j sits at offset (spacing*i, spacing*j) pixels.  x sweeps over
    [xlo, xlo+xspan] at 'speed' pixels/sample (bouncing), plus the detector offset, wrapped modulo
    nxpix if wrap_x.  y = y0 + ydrift*t + offset, or, if yspeed is given, y bounces over
    [y0, y0+yspan] at 'yspeed' pixels/sample.
    """
    ndet = ndet_y * ndet_x
    xspan = (nxpix - 1) if xspan is None else xspan
    out = torch.empty((3, ndet, nt), dtype=dtype, device=device)
    t = torch.arange(nt, dtype=torch.float64, device=device)
    xs = xlo + triangle(speed * t, float(xspan))
    if yspeed is None:
        ys = y0 + ydrift * t
    else:
        ys = y0 + triangle(yspeed * t, float(yspan))
    # One detector row at a time keeps the float64 temporaries at (ndet_x, nt).
    j = torch.arange(ndet_x, dtype=torch.float64, device=device)[:, None]
    for i in range(ndet_y):
        d = ndet_x * i + j
        x = xs[None, :] + spacing * j
        if wrap_x:
            x = torch.remainder(x, float(nxpix))
        rows = slice(ndet_x * i, ndet_x * (i + 1))
        out[0, rows] = (ys[None, :] + spacing * i).to(dtype)
        out[1, rows] = x.to(dtype)
        frac = torch.remainder(t[None, :] / alpha_period + d / float(ndet), 1.0)
        out[2, rows] = (2.0 * math.pi * frac).to(dtype)
    return out


def _normal(shape, seed, device, dtype=torch.float32):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return torch.randn(shape, generator=g, device=device, dtype=dtype)


def config1(device="cpu", seed=0):
    """3x1024x2048 map ~N(0,1), all cells, periodic; 64 detectors (8x8, 3 px) x 65536 samples
    (nsamp = 2^22), x sweep 0.5 px/sample over 0..2047, y drift 1e-3 px/sample from 100."""
    ny, nx = 1024, 2048
    xp = raster_xpointing(8, 8, 65536, 3.0, 0.5, nx, 100.0, 1.0e-3, device=device)
    m = _normal((3, ny, nx), seed, device)
    tod = _normal((64, 65536), seed + 1, device)
    return dict(nypix=ny, nxpix=nx, periodic=True, xpointing=xp, map=m, tod=tod, name="cfg1")


def config2_xpointing(device="cuda", ndet_side=32, nt=2 ** 18):
    """xpointing of the large run: 1024 detectors (32x32, 2 px) x 2^18 samples (2^28), x sweep
    0.7 px/sample bouncing over 0..32767 (wrapped), y drift 2e-4 px/sample from y0 = 100."""
    return raster_xpointing(ndet_side, ndet_side, nt, 2.0, 0.7, 32768, 100.0, 2.0e-4, device=device)


def config3_xpointing(device="cuda", nt=2 ** 22):
    """High-hit patch: 64 detectors (8x8, 2 px) x 2^22 samples (2^28) confined to [256, 768)^2:
    x bounces at 0.7 px/sample, y at an incommensurate 0.0123 px/sample (~1000 hits/pixel)."""
    return raster_xpointing(8, 8, nt, 2.0, 0.7, 1024, 256.0, 0.0, xlo=256.0, xspan=511.0 - 14.0,
                            yspan=511.0 - 14.0, yspeed=0.0123, wrap_x=False, device=device)


def cells_of_plan(plan_mt):
    """Sorted unique (iycell, ixcell) pairs of a plan's mt words (numpy uint64 or torch int64)."""
    if isinstance(plan_mt, torch.Tensor):
        c = torch.unique(plan_mt & ((1 << 20) - 1)).cpu().numpy()
    else:
        c = np.unique(np.asarray(plan_mt).astype(np.uint64) & np.uint64((1 << 20) - 1)).astype(np.int64)
    return [(int(v) >> 10, int(v) & 1023) for v in c]


def rotated_raster(ndet_side, nt, spacing, speed, theta, x0, y0, xspan, yspan, yspeed, nxpix, alpha_period=4096.0,
                   device="cpu"):
    """xpointing (3, ndet_side^2, nt) float32 of a detector grid rotated by 'theta' about its first
    detector: x bounces over [x0, x0+xspan] at 'speed' px/sample, y over [y0, y0+yspan] at 'yspeed'."""
    ndet = ndet_side * ndet_side
    t = torch.arange(nt, dtype=torch.float64, device=device)
    xs = x0 + triangle(speed * t, float(xspan))
    ys = y0 + triangle(yspeed * t, float(yspan))
    i = torch.arange(ndet_side, dtype=torch.float64, device=device).repeat_interleave(ndet_side)
    j = torch.arange(ndet_side, dtype=torch.float64, device=device).repeat(ndet_side)
    c, s = math.cos(theta), math.sin(theta)
    oy = spacing * (c * i - s * j)
    ox = spacing * (s * i + c * j)
    out = torch.empty((3, ndet, nt), dtype=torch.float32, device=device)
    out[0] = (ys[None, :] + oy[:, None]).to(torch.float32)
    out[1] = (xs[None, :] + ox[:, None]).to(torch.float32)
    d = torch.arange(ndet, dtype=torch.float64, device=device)[:, None]
    out[2] = (2.0 * math.pi * torch.remainder(t[None, :] / alpha_period + d / float(ndet), 1.0)).to(torch.float32)
    return out


def config4_tods(device="cuda", ntod=64, seed=1000, median=2 ** 20, sigma=1.0, ny=4096, nx=8192, ndet_side=4):
    """The batched workload: 'ntod' TODs whose nsamp is lognormal (median 2^20, sigma 1.0), clipped to
    [2^16, 2^24] and rounded to a multiple of 32 * ndet; TOD i is seeded with seed + i: random start
    pixel, sweep speed U(0.3, 1.0) px/sample, random detector-grid rotation, inside an ny x nx map.
    Returns a list of xpointing tensors of shape (3, nsamp)."""
    out = []
    quantum = 32 * ndet_side * ndet_side
    for i in range(ntod):
        rng = np.random.default_rng(seed + i)
        nsamp = int(np.clip(np.exp(np.log(median) + sigma * rng.standard_normal()), 2 ** 16, 2 ** 24))
        nsamp = max(quantum, (nsamp // quantum) * quantum)
        nt = nsamp // (ndet_side * ndet_side)
        speed = rng.uniform(0.3, 1.0)
        theta = rng.uniform(0.0, 2.0 * math.pi)
        margin = 4.0 + 2.0 * ndet_side * 1.5
        xspan = rng.uniform(256.0, 2048.0)
        yspan = rng.uniform(16.0, 128.0)
        x0 = rng.uniform(margin, nx - margin - xspan - 1.0)
        y0 = rng.uniform(margin, ny - margin - yspan - 1.0)
        xp = rotated_raster(ndet_side, nt, 1.5, speed, theta, x0, y0, xspan, yspan, speed * 0.01, nx, device=device)
        out.append(xp.reshape(3, nsamp).contiguous())
    return out
