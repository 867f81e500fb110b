"""A serving loop for pointing operations with continuous batching (no counterpart in the reference).

PointingServer keeps a pool of TODs' pointing, a resident input map (read by map2tod) and an output
map (into which tod2map accumulates) on the device, and serves three kinds of requests:

  * ('plan', tod_id):    build the TOD's plan and keep it in the device plan cache;
  * ('map2tod', tod_id): the TOD's samples from the input map (a new device array per request: a
                         view into one allocation per launch);
  * ('tod2map', tod_id, tod): accumulate a TOD array into the output map.

A worker thread runs the loop.  Every iteration it

  1. takes the newly submitted requests and admits them in arrival order while their device memory
     (plans, output TODs, batch plans) fits the HBM budget, evicting least-recently-used plans that no
     admitted request needs; requests that do not fit wait and are admitted as memory frees up;
  2. launches the admitted work on one of several CUDA streams: the plans it needs (plan requests,
     and operator requests whose plan is not cached), all built together into single-TOD plans; then
     all admitted map2tod requests as one TodBatch whose plan is merged from the cached single-TOD
     plans, then all admitted tod2map requests likewise -- so requests that arrive while others are
     on the GPU join the next launch, and launches of successive iterations overlap (a launch of
     one TOD uses its cached plan as is).

A completion thread waits on each launch's CUDA event in launch order, completes its requests and
returns their memory to the budget, waking the worker for requests that wait for memory.

Streams: submit() records an event on the caller's current CUDA stream, and the launch that serves
the request waits for it before reading the request's TOD, the pointing or the resident maps, so
inputs written asynchronously by the caller are safe to submit.  A map2tod result is recorded on the
submitting stream (Tensor.record_stream), so the caching allocator does not hand its memory to a
later launch while work the caller queues on that stream may still read it; use it on other streams
only after ordering them after the submitting stream.

Errors: a request with bad arguments raises in submit().  Device error bits (the reference's
xpointing-range and pixelization errors) are read back per launch, and every request of a launch
that reported bits fails with a RuntimeError naming them (a launch batches several requests; the
bits are not attributed to one of them); check() raises if any launch reported bits since the last
check().

Results do not depend on the mix: map2tod evaluates every sample with the same rounded operations as
the single-TOD operator (bit-identical), and tod2map adds the same per-sample contributions into the
output map (float atomics: the order, and so the last bits, differ).

Latency of a request = completion time - submission time, on the host clock.
"""

import collections
import concurrent.futures
import threading
import time

import numpy as np
import torch

from . import gpu_mm_pybind11 as _m
from .batch import TodBatch


# Streams shared by every server of the process, per device: torch's caching allocator keeps freed
# device blocks per stream, so a server on streams of its own could not reuse what an earlier one
# freed, and each of its allocations (plans, output TODs) would go to cudaMalloc.
_STREAM_POOL = {}


def _server_streams(n):
    dev = torch.cuda.current_device()
    pool = _STREAM_POOL.setdefault(dev, [])
    while len(pool) < n:
        pool.append(torch.cuda.Stream())
    return pool[:n]


# Grow-only scratch per server stream (batch plans and their sort space, up to ~GBs for large
# iterations): allocated once and reused by every later iteration on that stream, which stream order
# makes safe.  Allocating them per iteration meant a cudaMalloc of that size each time (measured up to
# 0.2 s per iteration) because the buffers of iterations still in flight cannot be reused.
_SCRATCH = {}


def _scratch(stream, key, nbytes):
    d = _SCRATCH.setdefault(stream.cuda_stream, {})
    buf = d.get(key)
    if buf is None or buf.numel() < nbytes:
        size = max(int(nbytes), 2 * (buf.numel() if buf is not None else 0))
        with torch.cuda.stream(stream):
            buf = torch.empty(size, dtype=torch.uint8, device="cuda")
        d[key] = buf
    return buf


def release_scratch():
    """Frees the scratch buffers that servers share (batch plans and their sort space, kept per
    stream between servers).  Call it only while no PointingServer is running; later servers
    allocate the buffers again."""
    torch.cuda.synchronize()
    _SCRATCH.clear()


class PointingServer:
    def __init__(self, xpointings, in_map, out_map, local_pixelization, hbm_budget_bytes, nstreams=3,
                 max_batch=256, tuning=None):
        self.xpointings = dict(xpointings)                # tod_id -> (3, nsamp) CUDA tensor
        self.in_map, self.out_map = in_map, out_map
        self.lpix = local_pixelization
        self.budget = int(hbm_budget_bytes)
        self.tuning = tuning
        self.max_batch = max_batch
        self.streams = _server_streams(nstreams)
        self._next_stream = 0
        self._lock = threading.Lock()
        self._wake = threading.Condition(self._lock)   # signalled by submit() and close()
        # Held by whichever thread admits and launches: the worker, or submit() when it finds the
        # server idle and launches its request at once (no wait for the worker to wake up).
        self._launch_mutex = threading.Lock()
        self._submitted = collections.deque()
        self._waiting = collections.deque()
        self._inflight = collections.deque()               # (event, requests, bytes, keepalive, error words, n), launch order
        self._done = threading.Condition(self._lock)       # signalled when a launch is queued, and at exit
        self._freed = 0                                    # bytes released by completions, not yet in _used
        self._worker_done = False
        self._launching = False                            # admitted requests between queues (see drain)
        self._plans = collections.OrderedDict()            # tod_id -> (single TodBatch, ready event, nbytes)
        self._used = 0
        self._stop = False
        self.latencies = {"plan": [], "map2tod": [], "tod2map": []}
        self.samples_done = 0
        self.launches = 0
        self.direct_launches = 0                           # launches made by submit() on an idle server
        self.evictions = 0
        self.iterations = []                               # (requests launched, host seconds)
        self.errors = []
        self._err_bits = 0                                 # device error bits seen since the last check()
        self._pinned_free = []                             # pinned host words for per-launch error readback
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._completer = threading.Thread(target=self._complete_loop, daemon=True)
        self._thread.start()
        self._completer.start()

    # ---- client side ----

    def submit(self, kind, tod_id, tod=None):
        """Queues a request and returns a concurrent.futures.Future: None for 'plan' and 'tod2map', the
        TOD (a CUDA tensor shaped like the pointing's sample axes) for 'map2tod'.  The request is served
        after the work queued so far on the caller's current CUDA stream."""
        if kind not in ("plan", "map2tod", "tod2map"):
            raise ValueError(f"unknown request kind {kind}")
        if tod_id not in self.xpointings:
            raise KeyError(f"unknown tod_id {tod_id}")
        if kind == "tod2map":
            if tod is None:
                raise ValueError("tod2map needs a TOD array")
            want = tuple(self.xpointings[tod_id].shape[1:])
            if not isinstance(tod, torch.Tensor) or tuple(tod.shape) != want:
                raise ValueError(f"tod2map: TOD shape {tuple(getattr(tod, 'shape', ()))} does not match the "
                                 f"pointing's sample shape {want}")
            if tod.dtype != torch.float32 or not tod.is_cuda or not tod.is_contiguous() or tod.data_ptr() % 16:
                raise ValueError("tod2map: the TOD must be a contiguous, 16-byte aligned float32 CUDA tensor")
        stream = torch.cuda.current_stream()
        ready = torch.cuda.Event()
        ready.record(stream)
        fut = concurrent.futures.Future()
        req = {"kind": kind, "id": tod_id, "tod": tod, "t0": time.perf_counter(), "fut": fut, "ready": ready,
               "stream": stream}
        direct = False
        with self._lock:
            idle = not (self._submitted or self._waiting or self._launching or self._stop)
            if idle and self._launch_mutex.acquire(blocking=False):
                direct = True
                self.direct_launches += 1
                self._waiting.append(req)
                self._take_freed()
                self._launching = True
            else:
                self._submitted.append(req)
                self._wake.notify()
        if direct:
            # An idle server launches the request from the caller's thread (the same admission and
            # launch as the worker's); anything left waiting goes to the worker.
            try:
                self._launch()
            except Exception as e:   # _launch has failed the requests of that launch only
                self.errors.append(repr(e))
            finally:
                with self._lock:
                    self._launching = False
                    if self._waiting or self._submitted:
                        self._wake.notify()
                self._launch_mutex.release()
        return fut

    def _take_freed(self):
        # With self._lock and self._launch_mutex held: memory that completions released.
        self._used -= self._freed
        self._freed = 0

    def drain(self, timeout=60.0):
        """Waits until every submitted request has completed."""
        t_end = time.perf_counter() + timeout
        while time.perf_counter() < t_end:
            with self._lock:
                busy = bool(self._submitted or self._waiting or self._inflight or self._launching)
            if not busy:
                return
            time.sleep(0.0002)
        raise TimeoutError("PointingServer.drain: requests still pending")

    def close(self):
        with self._lock:
            self._stop = True
            self._wake.notify()
        self._thread.join()
        self._completer.join()
        torch.cuda.synchronize()
        # Release the plan cache and the launches' buffers now rather than when the server object is
        # collected, so that a later server's allocations can reuse the blocks.
        self._plans.clear()
        self._inflight.clear()
        self._used = 0

    def stats(self):
        out = {}
        for k, v in self.latencies.items():
            if v:
                a = np.asarray(v) * 1e3
                out[k] = {"n": len(v), "p50_ms": round(float(np.percentile(a, 50)), 3),
                          "p99_ms": round(float(np.percentile(a, 99)), 3)}
        allv = sum(self.latencies.values(), [])
        if allv:
            a = np.asarray(allv) * 1e3
            out["all"] = {"n": len(allv), "p50_ms": round(float(np.percentile(a, 50)), 3),
                          "p99_ms": round(float(np.percentile(a, 99)), 3)}
        out["launches"] = self.launches
        out["direct_launches"] = self.direct_launches
        out["evictions"] = self.evictions
        if self.iterations:
            it = np.asarray(self.iterations, dtype=np.float64)
            out["iterations"] = {"n": len(it), "mean_requests": round(float(it[:, 0].mean()), 2),
                                 "host_ms_mean": round(1e3 * float(it[:, 1].mean()), 3),
                                 "host_ms_max": round(1e3 * float(it[:, 1].max()), 3)}
        out["plan_cache"] = {"plans": len(self._plans), "bytes": self._used}
        return out

    # ---- memory accounting ----

    def _plan_nbytes(self, tod_id):
        n = self.xpointings[tod_id][0].numel()
        return 16 * (n // 32) + (1 << 17) + (1 << 20)    # plan (owner list + cell bitmap) + sort scratch

    def _request_nbytes(self, r):
        n = self.xpointings[r["id"]][0].numel()
        extra = 4 * n if r["kind"] == "map2tod" else 0
        return extra + 16 * (n // 32) + (1 << 18)                      # output TOD + its share of the batch plan

    def _evict(self, need, pinned):
        for tid in list(self._plans.keys()):
            if self._used + need <= self.budget:
                return True
            if tid in pinned:
                continue
            _, ev, nb = self._plans.pop(tid)
            ev.synchronize()
            self._used -= nb
            self.evictions += 1
        return self._used + need <= self.budget

    # ---- worker ----

    def _stream(self):
        s = self.streams[self._next_stream]
        self._next_stream = (self._next_stream + 1) % len(self.streams)
        return s

    def _run(self):
        try:
            while not self._stop:
                with self._launch_mutex:
                    with self._lock:
                        while self._submitted:
                            self._waiting.append(self._submitted.popleft())
                        self._take_freed()
                        self._launching = bool(self._waiting)
                    try:
                        launched = self._launch()
                    except Exception as e:   # _launch has failed the requests of that launch only
                        launched = False
                        self.errors.append(repr(e))
                    finally:
                        self._launching = False
                if not launched:
                    # Nothing to launch: sleep until a request arrives or a completion frees memory
                    # (requests waiting for memory also retry after a short timeout).
                    with self._lock:
                        if not (self._submitted or self._freed or self._stop):
                            self._wake.wait(timeout=0.005 if self._waiting else 0.05)
        finally:
            with self._lock:
                self._worker_done = True
                self._done.notify()

    def _complete_loop(self):
        """Completion thread: waits for the oldest launch's event (the wait releases the GIL), then
        completes its requests and hands the memory back to the worker.  Launches on different
        streams may finish out of order; a later one is then completed right after the earlier."""
        while True:
            with self._lock:
                while not self._inflight and not self._worker_done:
                    self._done.wait(timeout=0.05)
                if not self._inflight:
                    return
                ev, reqs, nb, keepalive, errs, nerr = self._inflight[0]
            err = None
            try:
                ev.synchronize()
                bits = 0
                for w in errs[:nerr].tolist():      # copied on the launch's stream before 'ev'
                    bits |= w
                if bits:
                    err = RuntimeError(f"PointingServer: device error bits {bits:#x} in a launch of "
                                       f"{len(reqs)} request(s) (1/2: xpointing y/x out of range, "
                                       f"8: not in LocalPixelization)")
            except Exception as e:
                bits = 0
                err = e
                self.errors.append(repr(e))
            t1 = time.perf_counter()
            with self._lock:
                self._inflight.popleft()
                self._freed += nb
                self._err_bits |= bits
                self._pinned_free.append(errs)
                for r in reqs:
                    self.latencies[r["kind"]].append(t1 - r["t0"])
                self._wake.notify()
            for r in reqs:
                if not r["fut"].done():
                    if err is None:
                        r["fut"].set_result(r.get("result"))
                    else:
                        r["fut"].set_exception(err)
            del keepalive

    def _launch(self):
        # A plan this iteration builds is reserved when its first request is admitted, so that the
        # admission of later requests in the same iteration sees it.
        admitted, pinned, reserved = [], set(), {}
        while self._waiting and len(admitted) < self.max_batch:
            r = self._waiting[0]
            new_plan = (r["id"] not in self._plans) and (r["id"] not in reserved)
            plan_nb = self._plan_nbytes(r["id"]) if new_plan else 0
            need = self._request_nbytes(r) + plan_nb
            pinned.add(r["id"])
            if not self._evict(need, pinned | {q["id"] for q in admitted}):
                pinned.discard(r["id"])
                break
            admitted.append(self._waiting.popleft())
            self._used += need
            if new_plan:
                reserved[r["id"]] = plan_nb
        if not admitted:
            return False
        try:
            t0 = time.perf_counter()
            ok = self._launch_admitted(admitted, reserved)
            self.iterations.append((len(admitted), time.perf_counter() - t0))
            return ok
        except Exception as e:
            # The admitted requests are no longer queued: fail them here so no client waits forever.
            for r in admitted:
                if not r["fut"].done():
                    r["fut"].set_exception(e)
                self._used -= self._request_nbytes(r)
            for tid, nb in reserved.items():
                if tid not in self._plans:
                    self._used -= nb
            raise

    def _pinned_words(self, n):
        with self._lock:
            for i, b in enumerate(self._pinned_free):
                if b.numel() >= n:
                    return self._pinned_free.pop(i)
        return torch.empty(max(n, 16), dtype=torch.int32, pin_memory=True)

    def _launch_admitted(self, admitted, reserved):
        stream = self._stream()
        keep = []
        errwords = []
        # Everything below is allocated and launched on 'stream', so allocations, copies and kernels
        # of one iteration are ordered, and iterations on different streams overlap.  It starts after
        # the work each request's caller had queued when submitting.
        for r in admitted:
            stream.wait_event(r["ready"])
        with torch.cuda.stream(stream):
            # Plans to (re)build: plan requests, and operator requests whose plan is not cached --
            # all built together (one owner pass, one sort, one scatter).
            need = []
            for r in admitted:
                if (r["kind"] == "plan" or r["id"] not in self._plans) and r["id"] not in need:
                    need.append(r["id"])
            if need:
                xps = [self.xpointings[i] for i in need]
                builder = TodBatch(xps, [x[0] for x in xps], self.lpix, tuning=self.tuning, upload_stream=stream,
                                   plan_buffers=False)
                lp = self.lpix
                tn = _m.batch_plan_each_tmp_nbytes(builder.total_lines, builder.ntod, lp.nypix_global,
                                                   lp.nxpix_global, builder.tuning)
                singles = builder.build_plans_each(stream, tmp=_scratch(stream, "each_tmp", tn))
                ev = torch.cuda.Event()
                ev.record(stream)
                for i, sp in zip(need, singles):
                    if i in self._plans:
                        self._used -= self._plans.pop(i)[2]
                    nb = max(self._plan_nbytes(i), sp.plan.numel())
                    self._plans[i] = (sp, ev, nb)
                    self._used += nb - reserved.get(i, 0)
                errwords.append(builder.err)
                keep.append(builder)
            for r in admitted:
                self._plans.move_to_end(r["id"])
            for kind in ("map2tod", "tod2map"):
                reqs = [r for r in admitted if r["kind"] == kind]
                if not reqs:
                    continue
                plans = [self._plans[r["id"]] for r in reqs]
                for ev in {id(p[1]): p[1] for p in plans}.values():
                    stream.wait_event(ev)
                xps = [self.xpointings[r["id"]] for r in reqs]
                if kind == "map2tod":
                    # One allocation per iteration, a view per request (16-byte aligned: nsamp is a
                    # multiple of 32); the block is freed when the last of its results is dropped.
                    sizes = [x[0].numel() for x in xps]
                    flat = torch.empty(sum(sizes), device="cuda")
                    tods = [v.view(x.shape[1:]) for v, x in zip(flat.split(sizes), xps)]
                    for r, t in zip(reqs, tods):
                        t.record_stream(r["stream"])
                        r["result"] = t
                else:
                    tods = [r["tod"] for r in reqs]
                b = TodBatch(xps, tods, self.lpix, tuning=self.tuning, upload_stream=stream, plan_buffers=False)
                if len(plans) == 1:
                    # One TOD: its cached plan is already the batch plan (a merge of one plan gives
                    # the same words).  The reference keeps it alive until the launch completes.
                    b.plan = plans[0][0].plan
                    b._merge_refs = [plans[0][0]]
                else:
                    pn, tn = _m.batch_plan_nbytes(b.total_lines, self.lpix.nypix_global, self.lpix.nxpix_global,
                                                  b.tuning)
                    b.use_buffers(_scratch(stream, "plan_" + kind, pn), _scratch(stream, "tmp_" + kind, tn))
                    b.merge_plans([p[0] for p in plans], stream)
                if kind == "map2tod":
                    b.map2tod(self.in_map, stream=stream)
                else:
                    b.tod2map(self.out_map, stream=stream)
                self.samples_done += b.total_samples
                self.launches += 1
                keep.append(b)
                errwords.append(b.err)
            # The launch's error words go to pinned host memory on the same stream, ahead of its event.
            dev = torch.cat(errwords) if len(errwords) > 1 else errwords[0]
            errs = self._pinned_words(dev.numel())
            errs[:dev.numel()].copy_(dev, non_blocking=True)
            keep.append(dev)
            ev = torch.cuda.Event()
            ev.record(stream)
        nb = sum(self._request_nbytes(r) for r in admitted)
        with self._lock:
            self._inflight.append((ev, admitted, nb, keep, errs, dev.numel()))
            self._done.notify()
        return True

    def check(self):
        """Waits for the submitted requests, then raises if any launch since the last check() reported
        device error bits (and clears them)."""
        self.drain()
        with self._lock:
            bits, self._err_bits = self._err_bits, 0
        if bits:
            raise RuntimeError(f"PointingServer: device error bits {bits:#x} since the last check()")
