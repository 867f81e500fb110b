"""Planned map2tod / tod2map over a TOD held in host memory, streamed to the GPU in chunks of
detectors so that host-to-device copies, plan builds, the operators and device-to-host copies
overlap.

No counterpart in the reference, whose operators take device arrays (gpu_mm.py:262-385) and leave
the copies to the caller.  A caller with TODs in host memory would otherwise copy the whole
xpointing and TOD, build the plan, run the operators and copy the result back one after another;
over PCIe the copies dominate, so here they run on their own streams while the GPU works on the
chunk before:

  streams 'h2d':    chunk i's xpointing rows (and TOD) into device slot i % nslots, on one of two
                    streams in turn (two copies in flight use PCIe better than one: 55 vs 49 GB/s)
  stream 'compute': chunk i's plan (a one-TOD batch plan: no host synchronisation), map2tod into the
                    slot's output TOD, tod2map from the slot's input TOD into the map
  stream 'd2h':     the slot's output TOD back into the host array

Events order the reuse of a slot (its inputs are overwritten only after the compute that read
them; its output only after the copy that drained it).  A chunk is a range of detectors: rows
[d0, d1) of each of the three (ndet, nt) planes of the xpointing, so every copy is contiguous.

Results: map2tod gives the bits of the planned operator (the same rounded arithmetic per sample);
tod2map adds the same per-sample contributions (float atomics, so the order of the additions, and
the last bits, differ).
"""

import torch

from . import gpu_mm_pybind11 as _m
from .batch import TodBatch
from .gpu_mm import LocalMap, LocalPixelization


def _host(t, name, shape):
    if not (isinstance(t, torch.Tensor) and t.device.type == "cpu" and t.dtype == torch.float32 and t.is_contiguous()):
        raise RuntimeError(f"HostPipeline: '{name}' must be a contiguous float32 CPU tensor")
    if not t.is_pinned():
        raise RuntimeError(f"HostPipeline: '{name}' must be in pinned memory (torch.empty(..., pin_memory=True)); "
                           "copies from pageable memory cannot overlap")
    if tuple(t.shape) != tuple(shape):
        raise RuntimeError(f"HostPipeline: '{name}' has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t


def _map_tensor(m, name):
    arr = m.arr if isinstance(m, LocalMap) else m
    if not (isinstance(arr, torch.Tensor) and arr.dtype == torch.float32 and arr.is_contiguous()):
        raise RuntimeError(f"HostPipeline: '{name}' must be a LocalMap or a contiguous float32 tensor")
    return arr


def chunk_plan(ndet, nt, chunk_dets=None, target_samples=1 << 24):
    """Detector ranges [(d0, d1), ...] covering range(ndet): about target_samples (or chunk_dets
    detectors) per chunk, every chunk a multiple of 32 samples.  Raises if ndet*nt is not."""
    ndet, nt = int(ndet), int(nt)
    if ndet <= 0 or nt <= 0 or (ndet * nt) % 32:
        raise RuntimeError(f"HostPipeline: ndet*nt = {ndet * nt} must be a positive multiple of 32")
    step = 1
    while (step * nt) % 32:
        step += 1                            # detectors per chunk must keep chunks a multiple of 32 samples
    cd = int(chunk_dets) if chunk_dets else max(1, target_samples // nt)
    cd = min(ndet, max(step, (cd // step) * step))
    chunks = [(d0, min(ndet, d0 + cd)) for d0 in range(0, ndet, cd)]
    # The last chunk holds ndet*nt - (whole chunks)*cd*nt samples: a multiple of 32 as both terms are.
    assert all(((d1 - d0) * nt) % 32 == 0 for d0, d1 in chunks)
    return cd, chunks


class HostPipeline:
    """Streams TODs of shape (ndet, nt) with pointing (3, ndet, nt) from pinned host memory through
    the planned operators against one LocalPixelization.

    chunk_dets: detectors per chunk (default: about 2^24 samples per chunk); rounded so that every
    chunk holds a multiple of 32 samples.  nslots: device buffers that chunks rotate through (3 lets
    one chunk copy in, one compute and one copy out at the same time).  Device memory: nslots chunks
    of xpointing + input TOD + output TOD (+ the maps, for host maps)."""

    def __init__(self, local_pixelization, ndet, nt, chunk_dets=None, nslots=3, tuning=None):
        if not isinstance(local_pixelization, LocalPixelization):
            raise RuntimeError("HostPipeline: expected a LocalPixelization")
        ndet, nt = int(ndet), int(nt)
        if nslots < 1:
            raise RuntimeError("HostPipeline: nslots must be >= 1")
        self.lpix = local_pixelization
        self.ndet, self.nt = ndet, nt
        cd, self.chunks = chunk_plan(ndet, nt, chunk_dets)
        self.chunk_dets = cd
        self.nslots = min(int(nslots), len(self.chunks))
        self.tuning = tuning
        n = cd * nt
        self._xp = [torch.empty(3 * n, dtype=torch.float32, device="cuda") for _ in range(self.nslots)]
        self._tin = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(self.nslots)]
        self._tout = [torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(self.nslots)]
        self._errs = torch.zeros((len(self.chunks), 3), dtype=torch.int32, device="cuda")
        self._batches = {}                   # (slot, ndet of chunk) -> (batch over tout, batch over tin)
        self._h2d = [torch.cuda.Stream(), torch.cuda.Stream()]
        self._comp, self._d2h = torch.cuda.Stream(), torch.cuda.Stream()
        self._free = [torch.cuda.Event() for _ in range(self.nslots)]      # compute done reading the slot
        self._drained = [torch.cuda.Event() for _ in range(self.nslots)]   # output copied out of the slot
        self._map_dev = {}
        self._partial = False
        self._pending = False
        for i, (d0, d1) in enumerate(self.chunks):   # batch descriptors are uploaded here, not in run()
            self._slot_batches(i % self.nslots, d1 - d0)
        torch.cuda.synchronize()

    def _slot_batches(self, k, nd):
        key = (k, nd)
        if key not in self._batches:
            n = nd * self.nt
            xp = self._xp[k][:3 * n].view(3, nd, self.nt)
            tout = self._tout[k][:n].view(nd, self.nt)
            tin = self._tin[k][:n].view(nd, self.nt)
            b = TodBatch([xp], [tout], self.lpix, tuning=self.tuning)
            self._batches[key] = (b, b.with_tods([tin]))
        return self._batches[key]

    def _device_map(self, key, m):
        buf = self._map_dev.get(key)
        if buf is None or buf.numel() != m.numel():
            buf = torch.empty(m.numel(), dtype=torch.float32, device="cuda")
            self._map_dev[key] = buf
        return buf

    def run(self, xpointing, map_in=None, tod_out=None, tod_in=None, map_out=None, partial_pixelization=False):
        """Queues the work and returns; wait() completes it and raises device errors.

        xpointing: (3, ndet, nt) pinned host array.  map2tod runs when 'tod_out' is given:
        tod_out (ndet, nt) pinned host <- map2tod(map_in).  tod2map runs when 'tod_in' is given:
        map_out += tod2map(tod_in).  Maps are LocalMaps or tensors of the pixelization's size, on the
        device (used in place) or in pinned host memory (copied in; map_out copied back as well)."""
        if self._pending:
            raise RuntimeError("HostPipeline.run: the previous run has not been waited for")
        ndet, nt = self.ndet, self.nt
        _host(xpointing, "xpointing", (3, ndet, nt))
        do_m2t, do_t2m = tod_out is not None, tod_in is not None
        if not (do_m2t or do_t2m):
            raise RuntimeError("HostPipeline.run: give tod_out (map2tod) and/or tod_in (tod2map)")
        if do_m2t:
            _host(tod_out, "tod_out", (ndet, nt))
            if map_in is None:
                raise RuntimeError("HostPipeline.run: map2tod needs map_in")
        if do_t2m:
            _host(tod_in, "tod_in", (ndet, nt))
            if map_out is None:
                raise RuntimeError("HostPipeline.run: tod2map needs map_out")
        self._partial = bool(partial_pixelization)
        cur = torch.cuda.current_stream()
        for s in (*self._h2d, self._comp, self._d2h):
            s.wait_stream(cur)               # inputs written on the caller's stream come first

        # Maps: host maps are copied in on the h2d stream before the first chunk.
        min_d = mout_d = mout_h = None
        if do_m2t:
            m = _map_tensor(map_in, "map_in")
            if m.is_cuda:
                min_d = m
            else:
                _host(m, "map_in", tuple(m.shape))
                min_d = self._device_map("in", m)
                with torch.cuda.stream(self._h2d[0]):
                    min_d.copy_(m, non_blocking=True)
        if do_t2m:
            m = _map_tensor(map_out, "map_out")
            if m.is_cuda:
                mout_d = m
            else:
                _host(m, "map_out", tuple(m.shape))
                mout_h = m
                mout_d = self._device_map("out", m)
                with torch.cuda.stream(self._h2d[0]):
                    mout_d.copy_(m, non_blocking=True)
        maps_in = torch.cuda.Event()
        maps_in.record(self._h2d[0])
        self._comp.wait_event(maps_in)

        for i, (d0, d1) in enumerate(self.chunks):
            k = i % self.nslots
            nd = d1 - d0
            n = nd * nt
            b_out, b_in = self._slot_batches(k, nd)
            # h2d: overwrite the slot once the compute that last read it is done.
            h2d = self._h2d[i % len(self._h2d)]
            h2d.wait_event(self._free[k])
            with torch.cuda.stream(h2d):
                xv = self._xp[k][:3 * n].view(3, nd, nt)
                for r in range(3):
                    xv[r].copy_(xpointing[r, d0:d1], non_blocking=True)
                if do_t2m:
                    self._tin[k][:n].view(nd, nt).copy_(tod_in[d0:d1], non_blocking=True)
            arrived = torch.cuda.Event()
            arrived.record(h2d)
            # compute: wait for the inputs, and for the copy that drained the slot's last output.
            self._comp.wait_event(arrived)
            self._comp.wait_event(self._drained[k])
            b_out.err = b_in.err = self._errs[i]
            b_out.build_plan(self._comp)
            if do_m2t:
                b_out.map2tod(min_d, partial_pixelization=self._partial, stream=self._comp)
            if do_t2m:
                b_in.tod2map(mout_d, partial_pixelization=self._partial, stream=self._comp)
            self._free[k].record(self._comp)
            # d2h: the slot's output back to the host.
            if do_m2t:
                self._d2h.wait_event(self._free[k])
                with torch.cuda.stream(self._d2h):
                    tod_out[d0:d1].copy_(self._tout[k][:n].view(nd, nt), non_blocking=True)
                self._drained[k].record(self._d2h)

        if mout_h is not None:
            done = torch.cuda.Event()
            done.record(self._comp)
            self._d2h.wait_event(done)
            with torch.cuda.stream(self._d2h):
                mout_h.copy_(mout_d, non_blocking=True)
        for s in (*self._h2d, self._comp, self._d2h):
            cur.wait_stream(s)
        self._pending = True

    def wait(self):
        """Waits for the queued run and raises the reference's error if a chunk reported one."""
        torch.cuda.synchronize()
        self._pending = False
        words = self._errs.cpu()
        if bool((words != 0).any()):
            ignore = 8 if self._partial else 0
            for i in range(words.shape[0]):
                for j in range(3):
                    if int(words[i, j]):
                        _m.errword_read(self._errs[i].data_ptr() + 4 * j, 0 if j == 0 else ignore, 0)
