"""Batches of TODs: one plan over many TODs and one launch per operator and stage.

No counterpart in the reference, which plans and applies one TOD per call (gpu_mm.py:1208-1299,
:262-385).  A TodBatch holds, per TOD, an xpointing array (3, nsamp) and a TOD array (nsamp,) or
(ndet, nt) -- torch CUDA float32, contiguous, 16-byte aligned, nsamp a multiple of 32 -- and one
LocalPixelization shared by all.  map2tod writes each TOD array; tod2map reads them.

  * build_plan(): one owner list over every cache line of every TOD, sorted by cell, plus the bitmap
    of cells touched.  Its size depends only on the number of cache lines, so nothing synchronises
    with the host and the build can be captured in a CUDA graph with the operators (capture()).
  * map2tod() / tod2map(): one launch each for the whole batch; a cell's tile is loaded once for
    every TOD that hits it.
  * Device error bits go to one word per stage; check() reads them and raises the reference's
    messages.

Results per TOD are those of the single-TOD planned operators (map2tod: the same arithmetic per
sample; tod2map: float atomics, so the summation order differs).
"""

import numpy as np
import torch

from . import gpu_mm_pybind11 as _m
from .gpu_mm import LocalMap, LocalPixelization

_DESC = np.dtype([("xpointing", "<u8"), ("tod", "<u8"), ("nsamp", "<i8"), ("line0", "<i8")])


def _stream_handle(stream):
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if isinstance(stream, torch.cuda.Stream) else int(stream)


def _check_pair(i, xp, tod):
    if not (isinstance(xp, torch.Tensor) and xp.is_cuda and xp.dtype == torch.float32 and xp.is_contiguous()):
        raise RuntimeError(f"TodBatch: xpointing[{i}] must be a contiguous float32 CUDA tensor")
    if not (isinstance(tod, torch.Tensor) and tod.is_cuda and tod.dtype == torch.float32 and tod.is_contiguous()):
        raise RuntimeError(f"TodBatch: tod[{i}] must be a contiguous float32 CUDA tensor")
    if xp.ndim not in (2, 3) or xp.shape[0] != 3:
        raise RuntimeError(f"TodBatch: xpointing[{i}] must have shape (3, nsamp) or (3, ndet, nt)")
    nsamp = xp[0].numel()
    if tuple(tod.shape) != tuple(xp.shape[1:]):
        raise RuntimeError(f"TodBatch: tod[{i}] shape {tuple(tod.shape)} does not match xpointing {tuple(xp.shape)}")
    if nsamp <= 0 or nsamp % 32 != 0:
        raise RuntimeError(f"TodBatch: TOD {i} has nsamp={nsamp}; must be a positive multiple of 32")
    if xp.data_ptr() % 16 or tod.data_ptr() % 16:
        raise RuntimeError(f"TodBatch: TOD {i}: xpointing and tod must be 16-byte aligned")
    return nsamp


class SinglePlan:
    """The plan of one TOD as a batch of one (owner list + cell bitmap), built by
    TodBatch.build_plans_each(); TodBatch.merge_plans() combines such plans."""

    def __init__(self, nsamp, lpix, tuning, stream=None):
        self.ntod = 1
        self.nsamp = int(nsamp)
        self.total_lines = self.nsamp // 32
        pn, _ = _m.batch_plan_nbytes(self.total_lines, lpix.nypix_global, lpix.nxpix_global, tuning)
        self.plan = torch.empty(pn, dtype=torch.uint8, device="cuda")


class TodBatch:
    """A batch of TODs against one LocalPixelization (see the module docstring).  With 'upload_stream'
    the descriptor table is copied to the device asynchronously on that stream (the batch must then
    be used on that stream); otherwise the copy completes before the constructor returns.
    plan_buffers=False skips the batch plan's buffers (for build_plans_each only)."""

    def __init__(self, xpointings, tods, local_pixelization, tuning=None, upload_stream=None, plan_buffers=True):
        if not isinstance(local_pixelization, LocalPixelization):
            raise RuntimeError("TodBatch: expected a LocalPixelization")
        if len(xpointings) != len(tods) or not (1 <= len(xpointings) <= 65535):
            raise RuntimeError("TodBatch: need 1..65535 (xpointing, tod) pairs")
        self.lpix = local_pixelization
        self.xpointings = list(xpointings)
        self.ntod = len(self.xpointings)
        self.nsamps = [_check_pair(i, x, t) for i, (x, t) in enumerate(zip(self.xpointings, tods))]
        self.total_samples = int(sum(self.nsamps))
        self.total_lines = self.total_samples // 32
        self.tuning = tuple(tuning) if tuning is not None else tuple(_m.batch_tuning_default())
        self.err = torch.zeros(3, dtype=torch.int32, device="cuda")   # build, map2tod, tod2map
        self._upload_stream = upload_stream
        self._set_tods(tods)
        if plan_buffers:            # not needed when the batch only builds single-TOD plans
            self._alloc()

    def _set_tods(self, tods):
        self.tods = list(tods)
        d = np.zeros(self.ntod, dtype=_DESC)
        d["xpointing"] = [x.data_ptr() for x in self.xpointings]
        d["tod"] = [t.data_ptr() for t in self.tods]
        d["nsamp"] = self.nsamps
        d["line0"] = np.concatenate([[0], np.cumsum(np.asarray(self.nsamps, np.int64) // 32)[:-1]])
        host = torch.from_numpy(d.view(np.uint8).copy())
        if self._upload_stream is None:
            self.descs = host.cuda()
            torch.cuda.current_stream().synchronize()
        else:
            self._descs_host = host.pin_memory()          # alive until the batch is dropped
            with torch.cuda.stream(self._upload_stream):
                self.descs = self._descs_host.cuda(non_blocking=True)

    def _alloc(self):
        pn, tn = _m.batch_plan_nbytes(self.total_lines, self.lpix.nypix_global, self.lpix.nxpix_global, self.tuning)
        self.plan = torch.empty(pn, dtype=torch.uint8, device="cuda")
        self.tmp = torch.empty(tn, dtype=torch.uint8, device="cuda")

    def with_tods(self, tods):
        """A batch over the same pointing (and the same plan buffers) with other TOD arrays."""
        b = object.__new__(TodBatch)
        b.__dict__.update(self.__dict__)
        for i, (x, t) in enumerate(zip(self.xpointings, tods)):
            _check_pair(i, x, t)
        b.err = torch.zeros(3, dtype=torch.int32, device="cuda")
        b._set_tods(tods)
        return b

    def merge_plans(self, singles, stream=None):
        """Builds this batch's plan from built single-TOD batches (TodBatch of one TOD each, in this
        batch's TOD order) instead of from the pointing: their owner lists are concatenated with the
        TOD index set, the cell bitmaps OR-ed and the list sorted by cell.  The result is the plan
        build_plan() gives."""
        if len(singles) != self.ntod or any(s.ntod != 1 or s.total_lines != n // 32
                                            for s, n in zip(singles, self.nsamps)):
            raise RuntimeError("TodBatch.merge_plans: need one single-TOD batch per TOD, with matching sizes")
        host = torch.tensor([[s.plan.data_ptr() for s in singles], [s.total_lines for s in singles]],
                            dtype=torch.int64).pin_memory()
        if isinstance(stream, torch.cuda.Stream) or stream is None:
            # Copy on the stream that runs the merge, so it is ordered before it.
            with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
                self._merge_args = host.cuda(non_blocking=True)
        else:
            self._merge_args = host.cuda()
            torch.cuda.current_stream().synchronize()
        self._merge_host = host            # kept alive until the next merge (the copy is asynchronous)
        self._merge_refs = list(singles)
        _m.batch_plan_merge(self._merge_args[0].data_ptr(), self._merge_args[1].data_ptr(), self.ntod,
                            self.total_lines, self.lpix.nypix_global, self.lpix.nxpix_global, self.plan.data_ptr(),
                            self.plan.numel(), self.tmp.data_ptr(), self.tmp.numel(), self.tuning,
                            _stream_handle(stream))

    def build_plans_each(self, stream=None, tmp=None):
        """The single-TOD plan of every TOD of the batch (a SinglePlan each), built together: one
        owner pass over all TODs, one sort by (TOD, cell), one scatter (at most 4096 TODs).  'tmp':
        optional uint8 CUDA scratch of at least batch_plan_each_tmp_nbytes bytes, used on 'stream'."""
        lp = self.lpix
        st = self._upload_stream if stream is None and self._upload_stream is not None else stream
        with torch.cuda.stream(st if isinstance(st, torch.cuda.Stream) else torch.cuda.current_stream()):
            singles = [SinglePlan(n, lp, self.tuning) for n in self.nsamps]
            ptrs = torch.tensor([sp.plan.data_ptr() for sp in singles], dtype=torch.int64).pin_memory()
            self._each_host = ptrs
            self._each_ptrs = ptrs.cuda(non_blocking=True)
            tn = _m.batch_plan_each_tmp_nbytes(self.total_lines, self.ntod, lp.nypix_global, lp.nxpix_global,
                                               self.tuning)
            if tmp is not None and tmp.numel() >= tn:
                self._each_tmp = tmp
            else:
                self._each_tmp = torch.empty(tn, dtype=torch.uint8, device="cuda")
        _m.batch_plan_build_each(self.descs.data_ptr(), self.ntod, self.total_lines, lp.nypix_global, lp.nxpix_global,
                                 bool(lp.periodic_xcoord), self._each_ptrs.data_ptr(), self._each_tmp.data_ptr(),
                                 self._each_tmp.numel(), self.tuning, self.err.data_ptr(), _stream_handle(st))
        return singles

    def use_buffers(self, plan, tmp):
        """Uses caller-owned uint8 CUDA buffers (at least batch_plan_nbytes each) for the batch plan
        and its scratch instead of allocating them; their users must be ordered (same stream)."""
        pn, tn = _m.batch_plan_nbytes(self.total_lines, self.lpix.nypix_global, self.lpix.nxpix_global, self.tuning)
        if plan.numel() < pn or tmp.numel() < tn:
            raise RuntimeError("TodBatch.use_buffers: buffers too small")
        self.plan, self.tmp = plan[:pn], tmp[:tn]

    def set_tuning(self, tuning):
        """Launch/sort parameters (sort_digit_bits, ctas_per_sm, min_lines_per_cta); the plan must be
        rebuilt afterwards."""
        self.tuning = tuple(int(v) for v in tuning)
        self._alloc()

    def build_plan(self, stream=None):
        _m.batch_plan_build(self.descs.data_ptr(), self.ntod, self.total_lines, self.lpix.nypix_global,
                            self.lpix.nxpix_global, bool(self.lpix.periodic_xcoord), self.plan.data_ptr(),
                            self.plan.numel(), self.tmp.data_ptr(), self.tmp.numel(), self.tuning,
                            self.err.data_ptr(), _stream_handle(stream))

    def map2tod(self, local_map, accum=False, partial_pixelization=False, stream=None):
        arr = local_map.arr if isinstance(local_map, LocalMap) else local_map
        _m.batch_map2tod(self.descs.data_ptr(), self.ntod, self.total_lines, arr, self.lpix, self.plan.data_ptr(),
                         partial_pixelization, accum, self.tuning, self.err.data_ptr() + 4, _stream_handle(stream))

    def tod2map(self, local_map, partial_pixelization=False, stream=None):
        arr = local_map.arr if isinstance(local_map, LocalMap) else local_map
        _m.batch_tod2map(self.descs.data_ptr(), self.ntod, self.total_lines, arr, self.lpix, self.plan.data_ptr(),
                         partial_pixelization, self.tuning, self.err.data_ptr() + 8, _stream_handle(stream))

    def check(self, partial_pixelization=False, stream=None):
        """Waits for 'stream' and raises if a stage reported device error bits."""
        s = _stream_handle(stream)
        _m.errword_read(self.err.data_ptr(), 0, s)
        ignore = 8 if partial_pixelization else 0
        _m.errword_read(self.err.data_ptr() + 4, ignore, s)
        _m.errword_read(self.err.data_ptr() + 8, ignore, s)

    def capture(self, fn):
        """Captures fn(stream_handle) -- e.g. lambda s: (b.build_plan(s), b.map2tod(m, stream=s)) -- in a
        CUDA graph after one uncaptured warm-up call; returns the torch.cuda.CUDAGraph."""
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn(side.cuda_stream)
        torch.cuda.current_stream().wait_stream(side)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn(torch.cuda.current_stream().cuda_stream)
        return g
