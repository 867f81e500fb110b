#!/usr/bin/env python
"""Benchmark of the pointing-operator hot path (planned map2tod + tod2map) on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--ndet-rows R]

Workload (default): the large plain GPU run -- 1024 detectors x 2^18 samples (nsamp = 2^28) of a
synthetic raster scan (0.7 px/sample x sweep, 2e-4 px/sample y drift, 32x32 detector grid at 2 px)
into a 3x8192x32768 periodic map whose LocalPixelization holds only the cells the scan hits.

A step is one planned map2tod followed by one planned tod2map over all samples, with the plan built
once beforehand and reused (the reference's plan-reuse loop).  value = samples processed by the
step (per GPU, times the number of GPUs) / device time of the step, in Gsamples/s.  The 4 GiB of
xpointing + TOD streamed per step is larger than L2, so no flush is needed between steps.

Other numbers on the JSON line:
  roofline     the dominant kernel's algorithmic bytes per launch / its CUDA-event duration, against
               the measured HBM copy bandwidth (MEASURED_PEAKS.json)
  rooflines    the same for both planned kernels
  e2e          the same metric through the public API from pinned HOST buffers: H2D of xpointing,
               TOD and map, preplan + plan, map2tod, tod2map, D2H of the TOD and map results
  cpu_baseline the reference's CPU operators (oracle/_ref: the reference header; else the oracle
               port) on all host cores over the same workload
  clocks       NVML SM clock samples during the timed region
  batched      64 uneven TODs (lognormal nsamp) into one map: plain per-TOD calls against one
               autotuned TodBatch replayed as CUDA graphs; speed-up, bitwise map2tod equality and
               tod2map error against the FP64 oracle
  served       Poisson request stream (plan / map2tod / tod2map) through PointingServer (continuous
               batching) and through sequential plain calls: p50/p99 latency, saturated Gsamples/s,
               bitwise map2tod equality, tod2map error against the FP64 oracle
  precision    tod2map precision variants (float atomics, compensated float flush, float64 map) on
               the high-hit workload (2^28 samples in a 512x512 box, tod = 1e3 + N(0,1)): throughput
               and max/rms relative error against the FP64 oracle on the host cores

N > 1 (torchrun): every rank runs its own replica of the workload on its own GPU (weak scaling, no
data-path collective); the step time is the max over ranks.  --impl reference runs the CPU
reference on rank 0 only.
"""

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gsamples/s map2tod+tod2map, % HBM peak; batched/served vs plain at stated err"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--ndet-rows", type=int, default=32, help="detector rows (32 = full 2^28-sample workload)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-precision", action="store_true", help="skip the tod2map precision study")
    p.add_argument("--no-batch", action="store_true", help="skip the batched-TOD study")
    p.add_argument("--no-serve", action="store_true", help="skip the serving study")
    p.add_argument("--only", default="", help="profiling aid: 'map2tod' or 'tod2map' runs only that operator")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def workload_config(ndet_rows, nsamp, ncells, npix):
    return {
        "workload": f"raster scan {ndet_rows}x32 detectors x 2^18 samples (nsamp={nsamp}), map 3x8192x32768 "
                    f"periodic, LocalPixelization = {ncells} hit cells (npix={npix})",
        "nsamp_per_gpu": nsamp,
        "step": "planned map2tod + planned tod2map, plan reused",
        "l2": "no flush: inputs (16 B/sample streamed, > 126 MB L2) exceed L2",
        "parallelism": "replicas (one TOD per GPU, weak scaling)",
    }


class ClockSampler:
    """Samples SM clock and clock-event reasons with NVML while the timed region runs."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
        0x100: "display_clock_setting",
    }

    def __init__(self, device_index):
        self.ok = False
        self.samples, self.reasons = [], set()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
                r = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["nvml unavailable"]}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons - {"gpu_idle"}), "n_samples": len(self.samples)}


# ------------------------------------------------------------------------------------------------


def cpu_reference_run(xp, tod, m, lp, nthreads, use_ref):
    import numpy as np
    import oracle
    out_tod = np.zeros_like(tod)
    out_map = np.zeros_like(m)
    t0 = time.perf_counter()
    e1 = oracle.map2tod_mt(out_tod, m, xp, lp, nthreads, use_ref=use_ref)
    e2 = oracle.tod2map_mt(out_map, tod, xp, lp, nthreads, use_ref=use_ref)
    dt = time.perf_counter() - t0
    assert e1 == 0 and e2 == 0
    return dt


def _synthetic():
    """gpu_mm_b200/synthetic.py (the seeded raster generator; it imports only numpy and torch), loaded
    from its file so that the CPU legs never run the package's __init__ and never map its native
    library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bench_synthetic", os.path.join(ROOT, "gpu_mm_b200", "synthetic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def cpu_sample(ndet, ndet_rows_cfg):
    """The first 'ndet' detectors of the workload, on the host: xpointing, tod, map, oracle Lpix."""
    import numpy as np
    import torch
    import oracle
    synthetic = _synthetic()
    rows = max(1, ndet // 32)
    xp = synthetic.raster_xpointing(rows, 32, 2 ** 18, 2.0, 0.7, 32768, 100.0, 2.0e-4, device="cpu").numpy()
    xp = np.ascontiguousarray(xp[:, :ndet])
    mt, _, err = oracle.plan(xp, 8192, 32768, True)
    cells = sorted({(int(c) >> 10, int(c) & 1023) for c in np.unique(mt & np.uint64(0xFFFFF))})
    offs = np.full((128, 512), -1, dtype=np.int64)
    for i, (a, b) in enumerate(cells):
        offs[a, b] = 3 * 4096 * i
    lp = oracle.Lpix(8192, 32768, offs, 64, 4096, True)
    g = torch.Generator().manual_seed(0)
    m = torch.randn(3 * lp.npix, generator=g).numpy()
    tod = torch.randn(xp.shape[1:], generator=g).numpy()
    return xp, tod, m, lp


def cpu_baseline(ndet_rows):
    import oracle
    use_ref = oracle.ref_available()
    nthreads = os.cpu_count() or 1
    ndet = 32 * ndet_rows               # the whole workload, as the reference arm
    xp, tod, m, lp = cpu_sample(ndet, ndet_rows)
    nsamp = xp.size // 3
    cpu_reference_run(xp, tod, m, lp, nthreads, use_ref)   # warm
    dt = min(cpu_reference_run(xp, tod, m, lp, nthreads, use_ref) for _ in range(3))
    # The reference's operators as it runs them (single-threaded, gpu_mm.hpp:227-228), on one core:
    # the first 64 detectors (2^24 samples).
    xp1, tod1, m1, lp1 = cpu_sample(64, ndet_rows)
    n1 = xp1.size // 3
    dt1 = min(cpu_reference_run(xp1, tod1, m1, lp1, 1, use_ref) for _ in range(2))
    return {"value": round(nsamp / dt / 1e9, 4), "unit": "Gsamples/s", "cores": nthreads,
            "kind": "reference" if use_ref else "port",
            "sample": f"{ndet} detectors ({nsamp} samples), map2tod + tod2map, "
                      f"best of 3, {nthreads} threads",
            "single_core": {"value": round(n1 / dt1 / 1e9, 4), "unit": "Gsamples/s", "cores": 1,
                            "sample": f"the first 64 detectors ({n1} samples), map2tod + tod2map, best of 2"}}


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    use_ref = oracle.ref_available()
    nthreads = os.cpu_count() or 1
    # The whole workload: the multi-threaded CPU tod2map has a fixed cost (a private map per thread,
    # zeroed and reduced), which a sample of it would make dominate.
    ndet = 32 * args.ndet_rows
    xp, tod, m, lp = cpu_sample(ndet, args.ndet_rows)
    nsamp = xp.size // 3
    for _ in range(args.warmup):
        cpu_reference_run(xp, tod, m, lp, nthreads, use_ref)
    times = [cpu_reference_run(xp, tod, m, lp, nthreads, use_ref) for _ in range(args.steps)]
    dt = sum(times) / len(times)
    value = nsamp / dt / 1e9
    kind = "reference" if use_ref else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Gsamples/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.ndet_rows, 2 ** 18 * 32 * args.ndet_rows, len(lp.cell_offsets[lp.cell_offsets >= 0]), lp.npix),
        "cpu_baseline": {"value": round(value, 4), "unit": "Gsamples/s", "cores": nthreads, "kind": kind,
                         "sample": f"{ndet} detectors ({nsamp} samples) per step, map2tod + tod2map, "
                                   f"{nthreads} threads"},
        "e2e": {"value": round(value, 4), "unit": "Gsamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu": reference_gpu_times(args.ndet_rows, lp),
    }
    print(json.dumps(line), flush=True)


def reference_gpu_times(ndet_rows, lp):
    """The reference's own plan builder and GPU operators (its src_lib sources compiled unchanged for
    sm_100a in oracle/_ref) on the same workload and GPU, timed with CUDA events around each call of
    its C++ API (which waits for its error-flag readback, as the reference always does).  None where
    that comparator was not built or there is no GPU."""
    import torch
    import oracle
    if not (oracle.refgpu_available() and torch.cuda.is_available()):
        return None
    synthetic = _synthetic()
    xp = synthetic.raster_xpointing(ndet_rows, 32, 2 ** 18, 2.0, 0.7, 32768, 100.0, 2.0e-4, device="cuda")
    nsamp = xp.numel() // 3
    offs_gpu = torch.from_numpy(lp.cell_offsets).cuda()
    gen = torch.Generator(device="cuda").manual_seed(1234)
    m = torch.randn(3 * lp.npix, generator=gen, device="cuda")
    tod_in = torch.randn(nsamp, generator=gen, device="cuda")
    tod_out = torch.empty(nsamp, device="cuda")
    map_out = torch.zeros(3 * lp.npix, device="cuda")
    errflags = torch.zeros(2048, dtype=torch.int32, device="cuda")

    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    plans = []
    out = {"plan_build_ms": round(timed(lambda: plans.append(oracle.RefGpuPlan(xp, 8192, 32768, True))), 4)}
    plan = plans[-1]
    del plans[:-1]
    out["planned_map2tod_ms"] = round(timed(lambda: plan.map2tod(tod_out, m, xp, lp, offs_gpu)), 4)
    out["planned_tod2map_ms"] = round(timed(lambda: plan.tod2map(map_out, tod_in, xp, lp, offs_gpu)), 4)
    out["unplanned_map2tod_ms"] = round(timed(lambda: oracle.refgpu_unplanned_map2tod(tod_out, m, xp, lp, offs_gpu, errflags)), 4)
    out["unplanned_tod2map_ms"] = round(timed(lambda: oracle.refgpu_unplanned_tod2map(map_out, tod_in, xp, lp, offs_gpu, errflags)), 4)
    step = out["planned_map2tod_ms"] + out["planned_tod2map_ms"]
    out["step_ms"] = round(step, 4)
    out["value"] = round(nsamp / (step * 1e-3) / 1e9, 3)
    out["unit"] = "Gsamples/s (planned map2tod + tod2map, plan reused)"
    out["plan_nmt"] = plan.plan_nmt
    out["build"] = "reference src_lib compiled unchanged for sm_100a against oracle/ksgpu_shim (oracle/Makefile)"
    return out


def precision_study(max_run_lines=32):
    """tod2map precision variants on the high-hit workload: 64 detectors x 2^22 samples (2^28)
    confined to the 512x512 box [256, 768)^2 of a 3x1024x1024 map (~1000 hits/pixel), tod = 1e3 +
    N(0,1).  Each mode is timed with CUDA events (3 calls after 1 warm-up) and compared with the FP64
    oracle (reference_tod2map<double> on the float32 inputs widened) on the host cores."""
    import numpy as np
    import torch
    import oracle
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    ny = nx = 1024
    xp = synthetic.config3_xpointing(device="cuda")
    nsamp = xp.numel() // 3
    gen = torch.Generator(device="cuda").manual_seed(3)
    tod = 1e3 + torch.randn(xp.shape[1:], generator=gen, device="cuda")
    pp = g.PointingPrePlan(xp, ny, nx, periodic_xcoord=False)
    plan = g.PointingPlan(pp, xp)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    n = 3 * lp.npix
    f32 = torch.zeros(n, device="cuda")
    comp = torch.zeros(n, device="cuda")
    f64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    lmap = g.LocalMap(lp, f32)
    calls = {
        "fp32_atomics": lambda: g.tod2map(lmap, tod, xp, plan),
        "fp32_compensated_flush": lambda: (g.tod2map_compensated(lmap, comp, tod, xp, plan, max_run_lines=max_run_lines),
                                           g.fold_compensation(lmap, comp)),
        "fp64_map": lambda: g.tod2map_f64(f64, lp, tod, xp, plan, max_run_lines=max_run_lines),
        # The same two modes with partials of up to 8x as many lines: fewer flushes, longer float sums.
        "fp32_compensated_flush_long_runs": lambda: (
            g.tod2map_compensated(lmap, comp, tod, xp, plan, max_run_lines=8 * max_run_lines),
            g.fold_compensation(lmap, comp)),
        "fp64_map_long_runs": lambda: g.tod2map_f64(f64, lp, tod, xp, plan, max_run_lines=8 * max_run_lines),
    }
    results = {}
    for name, fn in calls.items():
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        f32.zero_()
        comp.zero_()
        f64.zero_()
        fn()
        torch.cuda.synchronize()
        out = (f64 if name.startswith("fp64_map") else f32).cpu().numpy().astype(np.float64)
        results[name] = {"ms": round(ms, 4), "gsamples_s": round(nsamp / (ms * 1e-3) / 1e9, 3), "out": out}
        if name.endswith("_long_runs"):
            results[name]["max_run_lines"] = 8 * max_run_lines
    xp_h = xp.cpu().numpy()
    tod_h = tod.cpu().numpy()
    want = np.zeros(n, np.float64)
    nthreads = os.cpu_count() or 1
    t0 = time.perf_counter()
    assert oracle.tod2map_f64w_mt(want, tod_h, xp_h, oracle.Lpix.rectangle(ny, nx, False), nthreads) == 0
    oracle_s = time.perf_counter() - t0
    for name, r in results.items():
        d = r.pop("out") - want
        r["max_rel_err"] = float(f"{np.abs(d).max() / np.abs(want).max():.3e}")
        r["rms_rel_err"] = float(f"{np.sqrt((d * d).sum() / (want * want).sum()):.3e}")
    return {
        "workload": "64 detectors x 2^22 samples (2^28) in the 512x512 box of a 3x1024x1024 map, ~1000 hits/pixel, "
                    "tod = 1e3 + N(0,1)",
        "error_metric": "max_rel = max|a-b| / max|b|, rms_rel = sqrt(sum (a-b)^2 / sum b^2), all three planes, "
                        "b = FP64 oracle (reference_tod2map<double> on the float32 inputs widened)",
        "max_run_lines": max_run_lines, "oracle_seconds": round(oracle_s, 2), "oracle_threads": nthreads,
        "modes": results,
    }


def hot_cells_study(max_run_lines=32):
    """float64 only in the high-hit cells, on a map with cells of very different depth: the high-hit
    TOD of the precision study (2^28 samples in the 512x512 box [256, 768)^2, ~1000 hits/pixel) and a
    shallow TOD over the whole 3x1024x1024 map (64 detectors x 2^20 samples, ~64 hits/pixel), both
    tod = 1e3 + N(0,1), accumulated into one map.  Modes: float atomics; a float64 map; float64 only
    in the cells touched by at least min_lines cache lines of the two plans (HotCells), folded into
    the float map once.  Times are CUDA events over both TODs (and the fold), mean of 3 after 1
    warm-up; errors against the FP64 oracle over the whole map and over the hot and the other cells."""
    import numpy as np
    import torch
    import oracle
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    ny = nx = 1024
    xd = synthetic.config3_xpointing(device="cuda")
    xw = synthetic.raster_xpointing(8, 8, 2 ** 20, 2.0, 0.7, nx, 0.0, 0.0, xlo=0.0, xspan=nx - 1.0 - 16.0,
                                    yspan=ny - 1.0 - 16.0, yspeed=0.0123, wrap_x=False, device="cuda")
    gen = torch.Generator(device="cuda").manual_seed(5)
    todos = []
    for xp in (xd, xw):
        tod = 1e3 + torch.randn(xp.shape[1:], generator=gen, device="cuda")
        pp = g.PointingPrePlan(xp, ny, nx, periodic_xcoord=False)
        todos.append((xp, tod, g.PointingPlan(pp, xp)))
    nsamp = sum(xp.numel() // 3 for xp, _, _ in todos)
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    n = 3 * lp.npix
    plans = [p for _, _, p in todos]
    lines = g.HotCells(lp, plans, 0).lines()
    min_lines = int(np.sqrt(float(np.median(lines)) * float(lines.max())))   # between the two depths
    hot = g.HotCells(lp, plans, min_lines)
    f32 = torch.zeros(n, device="cuda")
    f64 = torch.zeros(n, dtype=torch.float64, device="cuda")
    lmap = g.LocalMap(lp, f32)

    def run_hot():
        for xp, tod, plan in todos:
            g.tod2map_hot_f64(lmap, hot, tod, xp, plan, max_run_lines=max_run_lines)
        hot.fold(lmap)

    calls = {
        "fp32_atomics": lambda: [g.tod2map(lmap, tod, xp, plan) for xp, tod, plan in todos],
        "fp64_map": lambda: [g.tod2map_f64(f64, lp, tod, xp, plan, max_run_lines=max_run_lines)
                             for xp, tod, plan in todos],
        "fp64_hot_cells": run_hot,
    }
    want = np.zeros(n, np.float64)
    nthreads = os.cpu_count() or 1
    for xp, tod, _ in todos:
        assert oracle.tod2map_f64w_mt(want, tod.cpu().numpy(), xp.cpu().numpy(),
                                      oracle.Lpix.rectangle(ny, nx, False), nthreads) == 0
    hot_mask = np.repeat(np.repeat(hot.slots() >= 0, 64, axis=0), 64, axis=1)
    w3 = want.reshape(3, ny, nx)
    scale = np.abs(want).max()
    results = {}
    for name, fn in calls.items():
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        f32.zero_()
        f64.zero_()
        fn()
        torch.cuda.synchronize()
        out = (f64 if name == "fp64_map" else f32).cpu().numpy().astype(np.float64)
        d = np.abs(out.reshape(3, ny, nx) - w3)
        results[name] = {"ms": round(ms, 4), "gsamples_s": round(nsamp / (ms * 1e-3) / 1e9, 3),
                         "max_rel_err": float(f"{d.max() / scale:.3e}"),
                         "max_rel_err_hot_cells": float(f"{d[:, hot_mask].max() / scale:.3e}"),
                         "max_rel_err_other_cells": float(f"{d[:, ~hot_mask].max() / scale:.3e}")}
    return {
        "workload": "high-hit TOD (2^28 samples, ~1000 hits/pixel in [256, 768)^2) + shallow TOD over the whole "
                    "3x1024x1024 map (2^26 samples, ~64 hits/pixel), tod = 1e3 + N(0,1), one map",
        "min_lines": min_lines, "hot_cells": int(hot.nhot), "cells": int(lp.nycells * lp.nxcells),
        "hot_accumulator_bytes": int(hot.nhot) * 3 * 4096 * 8, "fp64_map_bytes": 8 * n,
        "max_run_lines": max_run_lines, "modes": results,
    }


def touched_cells(plan_bytes, total_lines):
    """(iycell, ixcell) of the cells set in a batch plan's cell bitmap (after the owner list)."""
    import numpy as np
    off = ((8 * total_lines + 127) // 128) * 128
    bits = np.unpackbits(plan_bytes[off:off + (1 << 17)].cpu().numpy(), bitorder="little")
    return [(int(c) >> 10, int(c) & 1023) for c in np.flatnonzero(bits)]


def fp64_oracle_cells(pairs, cells, ny, nx, periodic):
    """FP64 oracle tod2map (reference_tod2map<double> on the float32 inputs widened) of every
    (xpointing, tod) CUDA pair, in one multithreaded call, into a compact map of 'cells' (the cells
    the pairs touch): float64 [ncells][3][64][64]."""
    import numpy as np
    import oracle
    offs = np.full(((ny + 63) // 64, (nx + 63) // 64), -1, dtype=np.int64)
    for k, (cy, cx) in enumerate(cells):
        offs[cy, cx] = 3 * 4096 * k
    lp = oracle.Lpix(ny, nx, offs, 64, 4096, periodic)
    xp = np.concatenate([x.reshape(3, -1).cpu().numpy() for x, _ in pairs], axis=1)
    tod = np.concatenate([t.reshape(-1).cpu().numpy() for _, t in pairs])
    want = np.zeros(3 * 4096 * len(cells), np.float64)
    assert oracle.tod2map_f64w_mt(want, tod, np.ascontiguousarray(xp), lp, os.cpu_count() or 1) == 0
    return want.reshape(len(cells), 3, 64, 64)


def rect_cells(arr, cells, ny, nx):
    """The cells of a rectangular-layout map (3, ny, nx) as float64 [ncells][3][64][64]."""
    import numpy as np
    a = arr.reshape(3, ny, nx)
    return np.stack([a[:, 64 * cy:64 * cy + 64, 64 * cx:64 * cx + 64].cpu().numpy() for cy, cx in cells]).astype(np.float64)


def rel_errs(a, want):
    import numpy as np
    d = a - want
    return {"max_rel_err": float(f"{np.abs(d).max() / np.abs(want).max():.3e}"),
            "rms_rel_err": float(f"{np.sqrt((d * d).sum() / (want * want).sum()):.3e}")}


def batch_study(reps=3):
    """64 TODs of lognormal nsamp (median 2^20, sigma 1.0, clipped to [2^16, 2^24]), each its own
    rotated raster, into one 3x4096x8192 map: plan build + map2tod + tod2map of every TOD, (a) as
    plain per-TOD calls (PointingPrePlan, PointingPlan, map2tod per TOD, then tod2map per TOD) and
    (b) as a TodBatch, autotuned, as two CUDA-graph replays (plan build + map2tod; tod2map).  Both
    timed with CUDA events; throughput = samples of the batch / time of the whole stage pair."""
    import numpy as np
    import torch
    import oracle
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    ny, nx = 4096, 8192
    xps = synthetic.config4_tods(device="cuda")
    nsamps = [x.shape[1] for x in xps]
    total = int(sum(nsamps))
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    gen = torch.Generator(device="cuda").manual_seed(44)
    lmap = g.LocalMap(lp, torch.randn(3 * lp.npix, generator=gen, device="cuda"))
    tods_in = [torch.randn(n, generator=gen, device="cuda") for n in nsamps]
    out_plain = [torch.zeros(n, device="cuda") for n in nsamps]
    out_batch = [torch.zeros(n, device="cuda") for n in nsamps]
    map_plain = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    map_batch = torch.zeros(3 * lp.npix, device="cuda")

    def plain():
        plans = []
        for xp, to in zip(xps, out_plain):
            pl = g.PointingPlan(g.PointingPrePlan(xp, ny, nx, periodic_xcoord=False), xp)
            plans.append(pl)
            g.map2tod(to, lmap, xp, pl)
        for xp, ti, pl in zip(xps, tods_in, plans):
            g.tod2map(map_plain, ti, xp, pl)

    b_out = g.TodBatch(xps, out_batch, lp)
    scratch = torch.zeros(3 * lp.npix, device="cuda")
    best, cand_ms = g.autotune.autotune(b_out, lmap, scratch)
    b_in = b_out.with_tods(tods_in)
    graph1 = b_out.capture(lambda st: (b_out.build_plan(st), b_out.map2tod(lmap, stream=st)))
    graph2 = b_in.capture(lambda st: b_in.tod2map(map_batch, stream=st))

    def batched():
        graph1.replay()
        graph2.replay()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    plain_ms = timed(plain)
    batch_ms = timed(batched)
    b_out.check()
    b_in.check()
    map2tod_equal = all(torch.equal(a, b) for a, b in zip(out_plain, out_batch))
    # One clean tod2map of each path against the FP64 oracle.
    map_plain.arr.zero_()
    plain()
    map_batch.zero_()
    batched()
    torch.cuda.synchronize()
    cells = touched_cells(b_out.plan, b_out.total_lines)
    want = fp64_oracle_cells(list(zip(xps, tods_in)), cells, ny, nx, False)
    pe = rel_errs(rect_cells(map_plain.arr, cells, ny, nx), want)
    be = rel_errs(rect_cells(map_batch, cells, ny, nx), want)
    return {
        "workload": f"64 TODs, nsamp lognormal (median 2^20, sigma 1.0, clipped [2^16, 2^24]), total {total} samples, "
                    "rotated rasters, 3x4096x8192 map",
        "stage": "plan build + map2tod + tod2map of every TOD",
        "plain_ms": round(plain_ms, 3), "batched_ms": round(batch_ms, 3),
        "plain_gsamples_s": round(total / (plain_ms * 1e-3) / 1e9, 3),
        "batched_gsamples_s": round(total / (batch_ms * 1e-3) / 1e9, 3),
        "speedup": round(plain_ms / batch_ms, 3),
        "map2tod_bitwise_equal": bool(map2tod_equal),
        "tod2map_vs_fp64": {"plain": pe, "batched": be, "cells": len(cells)},
        "autotune": {"best": list(best), "candidates_ms": cand_ms},
    }


def serving_study(rate=200.0, duration_s=2.5, ntod_pool=128, seed=5):
    """Poisson arrivals at 'rate' req/s for 'duration_s' (seeded): 40% plan build, 30% map2tod, 30%
    tod2map, on TODs drawn uniformly from a pool of 'ntod_pool' TODs sized as the batched workload,
    against a resident 3x8192x32768 map; plan cache budget 120 GB.  (a) PointingServer (continuous
    batching) and (b) sequential plain calls (one request at a time, plans cached the same way) serve
    the same request stream at the same arrival times; latency = completion - arrival.  Then both
    serve the same requests all at once (saturated, best of five runs per arm): sustained
    Gsamples/s = samples processed / (last completion - first arrival).  Each arm first serves the
    burst and the Poisson stream once, untimed.  Results: map2tod of every request compared bitwise between
    (a) and (b); the tod2map output maps against the FP64 oracle."""
    import threading
    import numpy as np
    import torch
    import oracle
    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    ny, nx = 8192, 32768
    xps = synthetic.config4_tods(device="cuda", ntod=ntod_pool, seed=2000, ny=ny, nx=nx)
    pool = dict(enumerate(xps))
    lp = g.LocalPixelization.make_rectangle(ny, nx, False)
    gen = torch.Generator(device="cuda").manual_seed(55)
    in_map = torch.randn(3 * lp.npix, generator=gen, device="cuda")
    tods = {i: torch.randn(x.shape[1], generator=gen, device="cuda") for i, x in pool.items()}
    rng = np.random.default_rng(seed)
    t, reqs = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration_s:
            break
        u = rng.random()
        kind = "plan" if u < 0.4 else ("map2tod" if u < 0.7 else "tod2map")
        reqs.append((t, kind, int(rng.integers(0, ntod_pool))))
    torch.cuda.synchronize()

    def served(times):
        out_map = torch.zeros(3 * lp.npix, device="cuda")
        srv = g.PointingServer(pool, in_map, out_map, lp, hbm_budget_bytes=120 << 30)
        futs, t0 = [], time.perf_counter()
        for (ta, kind, i) in times:
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            futs.append((kind, i, srv.submit(kind, i, tod=tods[i] if kind == "tod2map" else None)))
        srv.drain(timeout=120)
        t_end = time.perf_counter()
        res = [(kind, i, f.result(timeout=60)) for kind, i, f in futs]
        srv.check()
        st = srv.stats()
        srv.close()
        return res, out_map, st, t_end - t0

    def sequential(times):
        out_map = torch.zeros(3 * lp.npix, device="cuda")
        lmap_in = g.LocalMap(lp, in_map)
        lmap_out = g.LocalMap(lp, out_map)
        plans, res, lat = {}, [], []
        t0 = time.perf_counter()
        for (ta, kind, i) in times:
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            xp = pool[i]
            if kind == "plan" or i not in plans:
                plans[i] = g.PointingPlan(g.PointingPrePlan(xp, ny, nx, periodic_xcoord=False), xp)
            r = None
            if kind == "map2tod":
                r = torch.empty(xp.shape[1], device="cuda")
                g.map2tod(r, lmap_in, xp, plans[i])
            elif kind == "tod2map":
                g.tod2map(lmap_out, tods[i], xp, plans[i])
            torch.cuda.synchronize()
            lat.append(time.perf_counter() - (t0 + ta))
            res.append((kind, i, r))
        return res, out_map, lat, time.perf_counter() - t0

    def pct(v):
        a = np.asarray(v) * 1e3
        return {"p50_ms": round(float(np.percentile(a, 50)), 3), "p99_ms": round(float(np.percentile(a, 99)), 3)}

    samples = sum(pool[i].shape[1] for _, _, i in reqs)
    burst = [(0.0, k, i) for _, k, i in reqs]
    # Warm-up of both arms (untimed), on the burst and on the Poisson stream: first launches of each
    # kernel, and the device and pinned host allocators' caches (the device allocator caches blocks
    # per stream, and the Poisson run's small launches land on the server's streams differently
    # from the burst's).
    served(burst)
    sequential(burst)
    served(reqs)
    sequential(reqs)
    res_a, map_a, st_a, _ = served(reqs)
    res_b, map_b, lat_b, _ = sequential(reqs)
    # Saturated: best of five for each arm (the server's host threads and the allocator make single
    # runs noisy: a host stall of a few hundred ms has been seen in one run).  Only the stats and wall
    # time of each run are kept, so a run's results and output map are freed before the next run
    # allocates its own.
    runs_a = [served(burst)[2:] for _ in range(5)]
    st_burst, wall_a = min(runs_a, key=lambda r: r[1])
    wall_b = min(sequential(burst)[3] for _ in range(5))
    m2t_equal = all(torch.equal(ra[2], rb[2]) for ra, rb in zip(res_a, res_b) if ra[0] == "map2tod")
    t2m = [(pool[i], tods[i]) for _, kind, i in reqs if kind == "tod2map"]
    probe = g.TodBatch([x for x, _ in t2m], [t for _, t in t2m], lp)
    probe.build_plan()
    cells = touched_cells(probe.plan, probe.total_lines)
    del probe
    want = fp64_oracle_cells(t2m, cells, ny, nx, False)
    return {
        "workload": f"Poisson {rate:g} req/s for {duration_s:g} s: {len(reqs)} requests (40% plan, 30% map2tod, "
                    f"30% tod2map) over a pool of {ntod_pool} TODs (nsamp lognormal, median 2^20), "
                    f"{samples} samples; resident 3x8192x32768 map; plan cache budget 120 GB",
        "served": {"latency": {k: v for k, v in st_a.items() if isinstance(v, dict) and "p50_ms" in v},
                   "launches": st_a["launches"]},
        "sequential_plain": {"latency": {"all": pct(lat_b)}},
        "saturated": {"served_gsamples_s": round(samples / wall_a / 1e9, 3),
                      "sequential_gsamples_s": round(samples / wall_b / 1e9, 3),
                      "speedup": round(wall_b / wall_a, 3), "served_wall_s": round(wall_a, 4),
                      "sequential_wall_s": round(wall_b, 4), "served_iterations": st_burst.get("iterations")},
        "map2tod_bitwise_equal": bool(m2t_equal),
        "tod2map_vs_fp64": {"served": rel_errs(rect_cells(map_a, cells, ny, nx), want),
                            "sequential_plain": rel_errs(rect_cells(map_b, cells, ny, nx), want), "cells": len(cells)},
    }


# ------------------------------------------------------------------------------------------------


def replica_throughput(local_ms, nsamp_per_rank, world, device):
    """Whole-job throughput of N independent replicas: every rank processed nsamp_per_rank samples,
    and the job took as long as its slowest rank (the max of the ranks' device-timed milliseconds,
    taken with one all-reduce).  Returns (max ms, Gsamples/s)."""
    import torch
    import torch.distributed as dist
    ms = float(local_ms)
    if world > 1:
        t = torch.tensor([ms], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, world * nsamp_per_rank / (ms * 1e-3) / 1e9


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return replica_throughput(x, 0, world, "cuda")[0]

    import gpu_mm_b200 as g
    from gpu_mm_b200 import synthetic
    peak, peak_kind = measured_peaks()

    # ---- workload (per rank: its own replica) ----
    xp = synthetic.raster_xpointing(args.ndet_rows, 32, 2 ** 18, 2.0, 0.7, 32768, 100.0 + rank, 2.0e-4, device="cuda")
    nsamp = xp.numel() // 3
    ny, nx = 8192, 32768

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pp = g.PointingPrePlan(xp, ny, nx)
    plan = g.PointingPlan(pp, xp)
    torch.cuda.synchronize()
    first_plan_s = time.perf_counter() - t0
    cells = synthetic.cells_of_plan(plan.get_plan_mt())
    lp = g.LocalPixelization.make_cells(ny, nx, cells)
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    lmap = g.LocalMap(lp, torch.randn(3 * lp.npix, generator=gen, device="cuda"))
    tod_in = torch.randn(xp.shape[1:], generator=gen, device="cuda")
    tod_out = torch.empty_like(tod_in)
    map_out = g.LocalMap(lp, torch.zeros(3 * lp.npix, device="cuda"))
    err_a = torch.zeros(1, dtype=torch.int32, device="cuda")
    err_b = torch.zeros(1, dtype=torch.int32, device="cuda")
    m = g.gpu_mm_pybind11

    # Plan build timing (preplan + plan into preallocated buffers), reused below.
    buf = torch.empty(pp.plan_nbytes, dtype=torch.uint8, device="cuda")
    tmp = torch.empty(pp.plan_constructor_tmp_nbytes, dtype=torch.uint8, device="cuda")
    nmt_buf = torch.empty(1024, dtype=torch.int32, device="cuda")
    pbuf = torch.empty(1024, dtype=torch.int32, device="cuda")
    plan_ms = []
    for i in range(4):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        pp2 = g.PointingPrePlan(xp, ny, nx, buf=nmt_buf, tmp_buf=pbuf)
        g.PointingPlan(pp2, xp, buf=buf, tmp_buf=tmp)
        e1.record()
        torch.cuda.synchronize()
        if i > 0:
            plan_ms.append(e0.elapsed_time(e1))

    do_m2t = args.only in ("", "map2tod")
    do_t2m = args.only in ("", "tod2map")

    def step(evs=None):
        if evs is not None:
            evs[0].record()
        if do_m2t:
            m.planned_map2tod_async(tod_out, lmap.arr, xp, lp, plan, False, False, err_a, 0)
        if evs is not None:
            evs[1].record()
        if do_t2m:
            m.planned_tod2map_async(map_out.arr, tod_in, xp, lp, plan, False, err_b, 0)
        if evs is not None:
            evs[2].record()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    m.check_errword(err_a, 0, 0)
    m.check_errword(err_b, 0, 0)

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        start.record()
        for k in range(args.steps):
            step(evs[k])
        stop.record()
        torch.cuda.synchronize()
    barrier()
    m.check_errword(err_a, 0, 0)
    m.check_errword(err_b, 0, 0)
    ms_step = max_over_ranks(start.elapsed_time(stop) / args.steps)
    m2t_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    t2m_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)

    npix = lp.npix
    m2t_bytes = 16 * nsamp + 12 * npix
    t2m_bytes = 16 * nsamp + 24 * npix
    dom = "tod2map" if t2m_ms >= m2t_ms else "map2tod"
    dom_ms, dom_bytes = (t2m_ms, t2m_bytes) if dom == "tod2map" else (m2t_ms, m2t_bytes)
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", f"{'planned_tod2map' if dom == 'tod2map' else 'planned_map2tod'}_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            td = json.load(f)
        traffic = int(td["bytes_per_sample"] * nsamp + td.get("bytes_per_pixel", 0) * npix)

    # Both planned kernels against the roofline (the dominant one is 'roofline' above).
    per_kernel = {}
    for kname, kms, kbytes in (("planned_map2tod", m2t_ms, m2t_bytes), ("planned_tod2map", t2m_ms, t2m_bytes)):
        kach = kbytes / (kms * 1e-3) / 1e9
        ktr = None
        kpath = os.path.join(ROOT, "profiles", f"{kname}_traffic.json")
        if os.path.exists(kpath):
            with open(kpath) as f:
                kd = json.load(f)
            ktr = int(kd["bytes_per_sample"] * nsamp + kd.get("bytes_per_pixel", 0) * npix)
        per_kernel[kname] = {"ms": round(kms, 4), "achieved_gbs": round(kach, 1), "frac": round(kach / peak, 4),
                             "algorithmic_bytes": kbytes, "traffic": ktr}

    # Unplanned operators (for context).
    unplanned = {}
    for name, fn in (("unplanned_map2tod_ms", lambda: m.unplanned_map2tod_async(tod_out, lmap.arr, xp, lp, False, False, err_a, 0)),
                     ("unplanned_tod2map_ms", lambda: m.unplanned_tod2map_async(map_out.arr, tod_in, xp, lp, False, err_b, 0))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            fn()
        e1.record()
        torch.cuda.synchronize()
        unplanned[name] = round(e0.elapsed_time(e1) / 3, 4)

    # ---- e2e through the public API from pinned host buffers ----
    e2e = None
    if not args.no_e2e:
        xp_h = torch.empty(xp.shape, dtype=torch.float32, pin_memory=True)
        xp_h.copy_(xp)
        tod_h = torch.empty(tod_in.shape, dtype=torch.float32, pin_memory=True)
        tod_h.copy_(tod_in)
        map_h = torch.empty(3 * npix, dtype=torch.float32, pin_memory=True)
        map_h.copy_(lmap.arr)
        tod_out_h = torch.empty_like(tod_h, pin_memory=True)
        map_out_h = torch.empty_like(map_h, pin_memory=True)
        xp_d = torch.empty_like(xp)
        tod_d = torch.empty_like(tod_in)
        map_d = torch.empty(3 * npix, dtype=torch.float32, device="cuda")
        out_tod_d = torch.empty_like(tod_in)
        out_map_d = torch.empty(3 * npix, dtype=torch.float32, device="cuda")

        def e2e_step():
            xp_d.copy_(xp_h, non_blocking=True)
            tod_d.copy_(tod_h, non_blocking=True)
            map_d.copy_(map_h, non_blocking=True)
            pre = g.PointingPrePlan(xp_d, ny, nx, buf=nmt_buf, tmp_buf=pbuf)
            pl = g.PointingPlan(pre, xp_d, buf=buf, tmp_buf=tmp)
            g.map2tod(out_tod_d, g.LocalMap(lp, map_d), xp_d, pl)
            out_map_d.zero_()
            g.tod2map(g.LocalMap(lp, out_map_d), tod_d, xp_d, pl)
            tod_out_h.copy_(out_tod_d, non_blocking=True)
            map_out_h.copy_(out_map_d, non_blocking=True)

        def timed_steps(fn, warm, k, post=None):
            for _ in range(warm):
                fn()
                torch.cuda.synchronize()
                if post:
                    post()
            barrier()
            ms = []
            for _ in range(k):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                torch.cuda.synchronize()
                if post:
                    post()
                ms.append(a.elapsed_time(b))
            barrier()
            return max_over_ranks(statistics.mean(ms))

        # The drop-in calls one after another: copies in, plan, operators, copies out.
        serial_ms = timed_steps(e2e_step, 1, 2)
        assert np.allclose(tod_out_h[0, :64].numpy(), tod_out[0, :64].cpu().numpy(), rtol=1e-5, atol=1e-5)

        # The same work through HostPipeline: chunks of detectors, copies in both directions on their
        # own streams, overlapping the per-chunk plans and operators.
        pipe = g.HostPipeline(lp, xp.shape[1], xp.shape[2])

        def pipe_step():
            out_map_d.zero_()
            pipe.run(xp_h, map_in=map_h, tod_out=tod_out_h, tod_in=tod_h, map_out=out_map_d)
            map_out_h.copy_(out_map_d, non_blocking=True)

        tod_out_h.fill_(float("nan"))
        e2e_ms = timed_steps(pipe_step, min(args.warmup, 3), max(1, min(args.steps, 5)), post=pipe.wait)
        assert torch.equal(tod_out_h, tod_out.cpu()), "pipelined map2tod differs from the device-timed run"
        hb = 4 * (xp.numel() + tod_in.numel() + 3 * npix)
        db = 4 * (tod_in.numel() + 3 * npix)
        e2e = {"value": round(world * nsamp / (e2e_ms * 1e-3) / 1e9, 4), "unit": "Gsamples/s",
               "h2d_bytes_per_step": hb, "d2h_bytes_per_step": db, "ms_per_step": round(e2e_ms, 3),
               "includes": "H2D xpointing+tod+map, plan, map2tod, tod2map, D2H tod+map (HostPipeline: "
                           f"{len(pipe.chunks)} chunks of {pipe.chunk_dets} detectors, copies overlapped)",
               "serial_drop_in": {"value": round(world * nsamp / (serial_ms * 1e-3) / 1e9, 4),
                                  "ms_per_step": round(serial_ms, 3),
                                  "includes": "the same through PointingPrePlan/PointingPlan/map2tod/tod2map, "
                                              "copies and calls one after another"}}
        del pipe

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.ndet_rows)
    def study(name, skip, fn):
        if rank != 0 or world != 1 or skip:
            return None
        t0 = time.perf_counter()
        r = fn()
        print(f"[bench] {name} study: {time.perf_counter() - t0:.1f} s", file=sys.stderr, flush=True)
        return r

    precision = study("precision", args.no_precision, precision_study)
    if precision is not None:
        precision["hot_cells"] = study("hot cells", False, hot_cells_study)
    batched = study("batched", args.no_batch, batch_study)
    served = study("serving", args.no_serve, serving_study)

    if rank == 0:
        value = world * nsamp / (ms_step * 1e-3) / 1e9
        step_bytes = (m2t_bytes if do_m2t else 0) + (t2m_bytes if do_t2m else 0)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Gsamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args.ndet_rows, nsamp, len(cells), npix),
            "pct_hbm_peak_step": round(100 * step_bytes / (ms_step * 1e-3) / 1e9 / peak, 2),
            "roofline": {"bound": "hbm", "kernel": f"planned_{dom}", "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                         "per_unit": "16 B/sample + 12 B/hit pixel (map2tod) or 24 B/hit pixel (tod2map)",
                         "frac_of_nominal_8tbs": round(achieved / 8000.0, 4)},
            "rooflines": per_kernel,
            "kernels_ms": {"planned_map2tod": round(m2t_ms, 4), "planned_tod2map": round(t2m_ms, 4),
                           **unplanned, "plan_build": round(statistics.mean(plan_ms), 4),
                           "first_plan_build_s": round(first_plan_s, 3)},
            "plan": {"nmt": int(pp.plan_nmt), "overhead": round(pp.overhead, 4), "sort_digit_bits": pp.sort_digit_bits},
            "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks.summary(), "precision": precision,
            "batched": batched, "served": served,
            "gpu_launches": args.steps * (int(do_m2t) + int(do_t2m)),
        }
        print(json.dumps(line), flush=True)

    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
