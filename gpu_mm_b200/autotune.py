"""Autotuner of the batched pointing operators.

Picks the radix digit width of the plan sort and the operator grid (CTAs per SM, minimum cache lines
per CTA slice) for a TodBatch by timing plan build + map2tod + tod2map with CUDA events over a
candidate grid.  Results are cached per batch shape (power-of-two bucket of the line count, the
number of TODs and the map geometry); pass 'cache_path' to keep them in a JSON file across runs.
"""

import itertools
import json
import os

import torch

_CACHE = {}


def default_candidates():
    return [(d, c, m) for d, c, m in itertools.product((4, 6, 8), (2, 4), (64, 256))]


def batch_key(batch):
    lines = max(1, int(batch.total_lines))
    ntod = max(1, int(batch.ntod))
    return (lines.bit_length(), ntod.bit_length(), int(batch.lpix.nypix_global), int(batch.lpix.nxpix_global),
            bool(batch.lpix.periodic_xcoord))


def _time(batch, map_in, map_out, reps):
    batch.build_plan()
    batch.map2tod(map_in)
    batch.tod2map(map_out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        batch.build_plan()
        batch.map2tod(map_in)
        batch.tod2map(map_out)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(batch, map_in, map_out, candidates=None, reps=2, cache_path=None):
    """Sets and returns the fastest tuning of 'batch' (sort_digit_bits, ctas_per_sm, min_lines_per_cta),
    with the per-candidate times in ms.  map_in / map_out are the local maps used for timing
    (map_out accumulates).  The batch's plan is rebuilt with the chosen tuning."""
    key = batch_key(batch)
    if cache_path and not _CACHE and os.path.exists(cache_path):
        with open(cache_path) as f:
            for k, v in json.load(f).items():
                _CACHE[tuple(json.loads(k))] = (tuple(v["best"]), v["times"])
    if key in _CACHE:
        best, times = _CACHE[key]
        batch.set_tuning(best)
        batch.build_plan()
        return best, times
    times = {}
    for cand in (candidates or default_candidates()):
        batch.set_tuning(cand)
        times[",".join(map(str, cand))] = round(_time(batch, map_in, map_out, reps), 4)
    best = tuple(int(v) for v in min(times, key=times.get).split(","))
    _CACHE[key] = (best, times)
    if cache_path:
        with open(cache_path, "w") as f:
            json.dump({json.dumps(list(k)): {"best": list(b), "times": t} for k, (b, t) in _CACHE.items()}, f)
    batch.set_tuning(best)
    batch.build_plan()
    return best, times
