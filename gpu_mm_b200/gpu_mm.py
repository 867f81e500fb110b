"""
Drop-in Python surface of gpu_mm's pointing operators, backed by hand-written sm_100a CUDA.

This mirrors kmsmith137/gpu_mm ``gpu_mm/gpu_mm.py`` for the pointing-operator path:

  map2tod(tod, local_map, xpointing, plan, partial_pixelization=False, response=None, debug=False, accum=False)
  tod2map(local_map, tod, xpointing, plan, partial_pixelization=False, response=None, debug=False)
  LocalPixelization, LocalMap, DynamicMap, PointingPrePlan, PointingPlan, read_xpointing_npzfile

with the same argument names, meanings and exceptions (gpu_mm.py:262-385, :421-806, :1208-1329).
Device arrays are torch CUDA tensors (any object with ``__cuda_array_interface__`` is accepted);
host arrays are numpy.  The reference used cupy, which is not part of this stack.

Data structures (see the reference's top-level docstring, gpu_mm.py:1-150):

* TOD: float32 ``tod[nsamp]`` or ``tod[ndet][nt]``; nsamp a multiple of 32 and <= 2^31.
* xpointing: float32 ``xpointing[3][nsamp]`` or ``[3][ndet][nt]``, rows {y, x, alpha}; a detector
  measures ``T + cos(2 alpha) Q + sin(2 alpha) U``.
* Local map: 64x64-pixel cells, element (pol, iy, ix) of cell (iycell, ixcell) at
  ``cell_offsets[iycell, ixcell] + pol*polstride + iy*ystride + ix``; negative offsets are absent cells.

The ``plan`` argument selects the operator: a PointingPlan (planned, fastest), None (unplanned), or
'reference' (the library's slow single-threaded CPU operator, for testing).  No path falls back
to the CPU silently; the package refuses to import without its native extension.
"""

import numpy as np
import torch

from . import gpu_mm_pybind11

mm_dtype = np.float64 if (gpu_mm_pybind11._get_tsize() == 8) else np.float32

_UNPLANNED_ERRFLAG_WORDS = 2048   # gpu_mm.py:306 ("max_blocks = 2048  # ad hoc")


def _device_zeros(n, dtype):
    return torch.zeros(n, dtype=dtype, device="cuda")


def map2tod(tod, local_map, xpointing, plan, partial_pixelization=False, response=None, debug=False, accum=False):
    """
    Arguments (gpu_mm.py:262-312):

      - tod: output array, shape (nsamp,) or (ndet, nt).  Overwritten unless accum=True.
      - local_map: input LocalMap.
      - xpointing: shape (3, nsamp) or (3, ndet, nt) array.
      - plan: a PointingPlan, None (plan-free GPU code), or 'reference' (CPU reference code).
      - partial_pixelization: if True, xpointing outside the local map reads zeros; if False, that
        raises an exception.
      - response: optional (2, ndet) per-detector (T, P) response; needs a PointingPlan.
      - accum: if True the result is added to 'tod'.
    """
    assert isinstance(local_map, LocalMap)
    lpix = local_map.pixelization
    larr = local_map.arr

    if isinstance(plan, PointingPlan):
        if response is None:
            gpu_mm_pybind11.planned_map2tod(tod, larr, xpointing, lpix, plan, partial_pixelization, debug, accum)
        else:
            gpu_mm_pybind11.response_map2tod(tod, larr, xpointing, response, lpix, plan, partial_pixelization, debug, accum)
    elif plan is None:
        errflag = _device_zeros(_UNPLANNED_ERRFLAG_WORDS, torch.int32)
        gpu_mm_pybind11.unplanned_map2tod(tod, larr, xpointing, lpix, errflag, partial_pixelization, accum)
    elif isinstance(plan, str) and plan == 'reference':
        gpu_mm_pybind11.reference_map2tod(tod, larr, xpointing, lpix, partial_pixelization, accum)
    else:
        raise RuntimeError(f"Bad 'plan' argument to map2tod(): {plan}")


def tod2map(local_map, tod, xpointing, plan, partial_pixelization=False, response=None, debug=False):
    """
    Arguments (gpu_mm.py:314-385):

      - local_map: output LocalMap or DynamicMap; tod2map() accumulates into it.
      - tod: input array, shape (nsamp,) or (ndet, nt).
      - xpointing: shape (3, nsamp) or (3, ndet, nt) array.
      - plan: a PointingPlan, None (plan-free GPU code), or 'reference' (CPU reference code).
      - partial_pixelization: as in map2tod().
      - response: optional (2, ndet) per-detector (T, P) response; needs a PointingPlan.
    """
    if isinstance(local_map, DynamicMap):
        if not isinstance(plan, PointingPlan):
            raise RuntimeError("tod2map(): if output is a DynamicMap, then the 'plan' argument"
                               + f" must be a PointingPlan (got: {plan})'")
        if partial_pixelization != local_map.have_cell_mask:
            raise RuntimeError(f"tod2map(): {partial_pixelization=} was specified,"
                               + f" but DynamicMap.have_cell_mask={local_map.have_cell_mask}"
                               + " (expected these to be equal)")
        local_map.expand(plan)
        if response is None:
            gpu_mm_pybind11.planned_tod2map(local_map._unstable_arr, tod, xpointing,
                                            local_map._unstable_pixelization, plan, partial_pixelization, debug)
        else:
            gpu_mm_pybind11.response_tod2map(local_map._unstable_arr, tod, xpointing, response,
                                             local_map._unstable_pixelization, plan, partial_pixelization, debug)
        return

    if not isinstance(local_map, LocalMap):
        raise RuntimeError(f"tod2map(): Bad 'local_map' argument to tod2map(): expected LocalMap or DynamicMap, got: {local_map}")

    lpix = local_map.pixelization
    larr = local_map.arr

    if isinstance(plan, PointingPlan):
        if response is None:
            gpu_mm_pybind11.planned_tod2map(larr, tod, xpointing, lpix, plan, partial_pixelization, debug)
        else:
            gpu_mm_pybind11.response_tod2map(larr, tod, xpointing, response, lpix, plan, partial_pixelization, debug)
    elif plan is None:
        errflag = _device_zeros(_UNPLANNED_ERRFLAG_WORDS, torch.int32)
        gpu_mm_pybind11.unplanned_tod2map(larr, tod, xpointing, lpix, errflag, partial_pixelization)
    elif isinstance(plan, str) and plan == 'reference':
        gpu_mm_pybind11.reference_tod2map(larr, tod, xpointing, lpix, partial_pixelization)
    else:
        raise RuntimeError(f"Bad 'plan' argument to tod2map(): {plan}")


####################################################################################################
#
# Precision variants of planned tod2map (no counterpart in the reference).  The samples are
# processed exactly as by tod2map() (float arithmetic, float partial sums per cell and row band, or
# per cell on the tile kernel); only the reduction of those partials into the map differs.


def tod2map_compensated(local_map, comp, tod, xpointing, plan, partial_pixelization=False, max_run_lines=0):
    """tod2map() into a float LocalMap whose float companion 'comp' (same size, zeroed before the
    first call) collects the rounding error of every float addition into the map (two-sum).
    local_map + comp then holds the sum to about twice float precision, across any number of calls;
    fold_compensation() adds comp into the map.  max_run_lines > 0 reduces each partial into the map
    after at most that many 32-sample cache lines."""
    if not isinstance(local_map, LocalMap) or not isinstance(plan, PointingPlan):
        raise RuntimeError("tod2map_compensated(): expected a LocalMap and a PointingPlan")
    gpu_mm_pybind11.planned_tod2map_compensated(local_map.arr, comp, tod, xpointing, local_map.pixelization, plan,
                                                partial_pixelization, int(max_run_lines))


def fold_compensation(local_map, comp):
    """Adds the compensation array of tod2map_compensated() into the map and zeroes it."""
    arr = local_map.arr if isinstance(local_map, LocalMap) else local_map
    gpu_mm_pybind11.fold_compensation(arr, comp)


class HotCells:
    """The high-hit cells of a LocalPixelization, for tod2map_hot_f64(): a cell is hot if at least
    'min_lines' 32-sample cache lines of the given plans touch it (counted over all of them).  Each
    hot cell gets a float64 accumulator (3 x 64 x 64 doubles) on the device, zero at construction;
    fold() adds the accumulators into a float LocalMap, rounding each value once, and zeroes them.
    Cells that are not hot take float atomics, as tod2map().  Rebuild it if the pixelization's
    cell_offsets change."""

    def __init__(self, local_pixelization, plans, min_lines):
        if not isinstance(local_pixelization, LocalPixelization):
            raise RuntimeError("HotCells(): expected a LocalPixelization")
        if isinstance(plans, PointingPlan):
            plans = [plans]
        plans = list(plans)
        if not all(isinstance(p, PointingPlan) for p in plans):
            raise RuntimeError("HotCells(): 'plans' must be PointingPlans")
        self.local_pixelization = local_pixelization
        self._h = gpu_mm_pybind11.HotCells(local_pixelization, plans, int(min_lines))

    @property
    def nhot(self):
        return self._h.nhot

    @property
    def min_lines(self):
        return self._h.min_lines

    def lines(self):
        """numpy (nycells, nxcells): cache lines of the plans touching each cell."""
        lp = self.local_pixelization
        return self._h.get_lines().reshape(lp.nycells, lp.nxcells)

    def slots(self):
        """numpy (nycells, nxcells): accumulator slot of each cell (in cell order), -1 if not hot."""
        lp = self.local_pixelization
        return self._h.get_slot().reshape(lp.nycells, lp.nxcells)

    def fold(self, local_map):
        """local_map += accumulators (one rounding per value); the accumulators become zero."""
        if not isinstance(local_map, LocalMap):
            raise RuntimeError("HotCells.fold(): expected a LocalMap")
        if local_map.pixelization is not self.local_pixelization:
            raise RuntimeError("HotCells.fold(): the LocalMap has another LocalPixelization")
        self._h.fold(local_map.arr, self.local_pixelization)


def tod2map_hot_f64(local_map, hot, tod, xpointing, plan, partial_pixelization=False, max_run_lines=0):
    """tod2map() into a float LocalMap in which the hot cells of 'hot' (a HotCells of the same
    LocalPixelization) reduce their partial sums with float64 atomics into their accumulators; call
    hot.fold(local_map) after the last TOD.  All other arithmetic is float, as in tod2map().  tod
    and xpointing must be 16-byte aligned."""
    if not isinstance(local_map, LocalMap) or not isinstance(plan, PointingPlan) or not isinstance(hot, HotCells):
        raise RuntimeError("tod2map_hot_f64(): expected a LocalMap, a HotCells and a PointingPlan")
    if local_map.pixelization is not hot.local_pixelization:
        raise RuntimeError("tod2map_hot_f64(): the LocalMap and the HotCells have different LocalPixelizations")
    gpu_mm_pybind11.planned_tod2map_hot_f64(local_map.arr, hot._h, tod, xpointing, local_map.pixelization, plan,
                                            partial_pixelization, int(max_run_lines))


def tod2map_f64(map64, local_pixelization, tod, xpointing, plan, partial_pixelization=False, max_run_lines=0):
    """tod2map() into a float64 map (contiguous, 3*npix doubles, laid out by 'local_pixelization'):
    float partials, reduced with double atomics."""
    if not isinstance(local_pixelization, LocalPixelization) or not isinstance(plan, PointingPlan):
        raise RuntimeError("tod2map_f64(): expected a LocalPixelization and a PointingPlan")
    gpu_mm_pybind11.planned_tod2map_f64(map64, tod, xpointing, local_pixelization, plan, partial_pixelization,
                                        int(max_run_lines))


####################################################################################################
#
# TOD preprocessing (gpu_mm.py:1420-1607 of the reference): deglitching, cut ranges, clip.
# Device arrays are torch CUDA tensors (float32 data, int32 index maps).


def get_border_means(out, signal, index_map):
    """Deglitching means on the GPU (gpu_mm.py:1423-1458): out[r] = (mean of signal[di, b00:b01],
    mean of signal[di, b10:b11]) for index_map[r] = (di, b00, b01, b10, b11); an empty range takes
    the other range's mean.  out (R,2) float32, signal (ndet,nt) float32, index_map (R,5) int32."""
    gpu_mm_pybind11.get_border_means(out, signal, index_map)


def deglitch(signal, bvals, index_map2):
    """Subtracts deglitching offsets on the GPU (gpu_mm.py:1461-1501), in place: with
    cumj = cumsum(bvals[:,1] - bvals[:,0]) and index_map2[r] = (di, r0, t1, t2),
    signal[di,t1:t2] = bvals[r,1] - dc and signal[di,t2:t3] -= dc, dc = cumj[r] - cumj[r0-1], t3 the
    next range's t1 if it has the same detector, else ntod."""
    gpu_mm_pybind11.deglitch(signal, bvals, None, index_map2)


def reference_get_border_means(signal, index_map):
    """CPU restatement of get_border_means() for testing (gpu_mm.py:1504-1529)."""
    R = len(index_map)
    bvals = np.zeros((R, 2), signal.dtype)
    for ri in range(R):
        di, b00, b01, b10, b11 = (int(v) for v in index_map[ri])
        a, b = signal[di, b00:b01], signal[di, b10:b11]
        v1 = np.mean(a) if a.size else 0.0
        v2 = np.mean(b) if b.size else 0.0
        bvals[ri] = (v1 if a.size else v2, v2 if b.size else v1)
    return bvals


def reference_deglitch(signal, bvals, index_map2):
    """CPU restatement of deglitch() for testing (gpu_mm.py:1532-1563); modifies 'signal'."""
    R, nsamp = len(index_map2), signal.shape[1]
    cumj = np.cumsum(bvals[:, 1] - bvals[:, 0])
    for ri in range(R):
        di, r0, t1, t2 = (int(v) for v in index_map2[ri])
        dcumj = cumj[ri] - (cumj[r0 - 1] if r0 > 0 else 0)
        last = not ((ri < R - 1) and (index_map2[ri + 1, 0] == di))
        t3 = nsamp if last else int(index_map2[ri + 1, 2])
        signal[di, t1:t2] = bvals[ri, 1] - dcumj
        signal[di, t2:t3] -= dcumj


def extract_ranges(tod, junk, offs, dets, starts, lens):
    """junk[offs[r] : offs[r]+lens[r]] = tod[dets[r], starts[r] : starts[r]+lens[r]] (gpu_mm.py:1593)."""
    gpu_mm_pybind11._ranges(0, tod, junk, offs, dets, starts, lens)


def insert_ranges(tod, junk, offs, dets, starts, lens):
    """tod[dets[r], starts[r] : starts[r]+lens[r]] = junk[offs[r] : offs[r]+lens[r]] (gpu_mm.py:1590)."""
    gpu_mm_pybind11._ranges(1, tod, junk, offs, dets, starts, lens)


def clear_ranges(tod, dets, starts, lens):
    """tod[dets[r], starts[r] : starts[r]+lens[r]] = 0 (gpu_mm.py:1596)."""
    gpu_mm_pybind11._ranges(2, tod, None, None, dets, starts, lens)


def clip(arr, vmin, vmax):
    """In-place clip of a float32 CUDA array (gpu_mm.py:1602-1607)."""
    gpu_mm_pybind11.clip(arr, float(vmin), float(vmax))


####################################################################################################


def _to_numpy_int64(a):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(a), dtype=np.int64)


class LocalPixelization(gpu_mm_pybind11.LocalPixelization):
    """
    Global pixelization (nypix_global, nxpix_global, periodic_xcoord) plus a set of 64x64 cells and
    their memory layout (cell_offsets, ystride, polstride); see gpu_mm.py:421-526.

    Members: nypix_global, nxpix_global, periodic_xcoord, cell_offsets_cpu (numpy),
    cell_offsets_gpu (torch), ystride, polstride, nycells, nxcells, npix.
    """

    def __init__(self, nypix_global, nxpix_global, cell_offsets, ystride, polstride, periodic_xcoord=True):
        self.cell_offsets_cpu = _to_numpy_int64(cell_offsets)
        self.cell_offsets_gpu = torch.as_tensor(self.cell_offsets_cpu).to("cuda")
        gpu_mm_pybind11.LocalPixelization.__init__(self, nypix_global, nxpix_global, self.cell_offsets_cpu,
                                                   self.cell_offsets_gpu, ystride, polstride, periodic_xcoord)

    def is_simple_rectangle(self):
        """True if the layout is a contiguous (3, 64*nycells, 64*nxcells) array (gpu_mm.py:450-458)."""
        rect_offsets = self._make_rectangular_cell_offsets(self.nycells, self.nxcells)
        return np.array_equal(self.cell_offsets_cpu, rect_offsets)

    def __eq__(self, x):
        assert isinstance(x, LocalPixelization)
        if self is x:
            return True
        if (self.nypix_global, self.nxpix_global) != (x.nypix_global, x.nxpix_global):
            return False
        if (self.periodic_xcoord, self.ystride, self.polstride) != (x.periodic_xcoord, x.ystride, x.polstride):
            return False
        if (self.nycells, self.nxcells, self.npix) != (x.nycells, x.nxcells, x.npix):
            return False
        return bool(np.all(np.maximum(self.cell_offsets_cpu, -1) == np.maximum(x.cell_offsets_cpu, -1)))

    __hash__ = None

    @classmethod
    def _make_rectangular_cell_offsets(cls, nycells, nxcells):
        cell_offsets = np.empty((nycells, nxcells), dtype=np.int64)
        cell_offsets[:, :] = 64 * np.arange(nxcells).reshape((1, -1))
        cell_offsets[:, :] += 64 * 64 * nxcells * np.arange(nycells).reshape((-1, 1))
        return cell_offsets

    @classmethod
    def make_rectangle(cls, nypix_global, nxpix_global, periodic_xcoord=True):
        """A LocalPixelization covering the whole global map as a contiguous
        (3, nypix_padded, nxpix_padded) array (gpu_mm.py:478-511)."""
        assert nypix_global > 0
        assert nxpix_global > 0
        nycells = (nypix_global + 63) // 64
        nxcells = (nxpix_global + 63) // 64
        return LocalPixelization(nypix_global, nxpix_global,
                                 cell_offsets=cls._make_rectangular_cell_offsets(nycells, nxcells),
                                 ystride=64 * nxcells, polstride=64 * 64 * nycells * nxcells,
                                 periodic_xcoord=periodic_xcoord)

    @classmethod
    def make_cells(cls, nypix_global, nxpix_global, cells, periodic_xcoord=True):
        """A LocalPixelization holding only the given cells (an iterable of (iycell, ixcell)), in
        cell-major layout float32[ncells][3][64][64] (ystride=64, polstride=64*64), in the given order."""
        nycells = (nypix_global + 63) // 64
        nxcells = (nxpix_global + 63) // 64
        offs = np.full((nycells, nxcells), -1, dtype=np.int64)
        for i, (iy, ix) in enumerate(cells):
            offs[iy, ix] = 3 * 64 * 64 * i
        return LocalPixelization(nypix_global, nxpix_global, offs, 64, 64 * 64, periodic_xcoord)


class LocalMap:
    """A LocalPixelization plus the map array 'arr' (torch CUDA tensor or numpy host array),
    float32 and contiguous (gpu_mm.py:529-580)."""

    def __init__(self, pixelization, arr):
        assert isinstance(pixelization, LocalPixelization)
        on_gpu = isinstance(arr, torch.Tensor) and arr.is_cuda
        assert on_gpu or isinstance(arr, np.ndarray), "LocalMap: 'arr' must be a torch CUDA tensor or a numpy array"
        if on_gpu:
            assert arr.dtype == torch.float32
            assert arr.is_contiguous()
        else:
            assert arr.dtype == np.float32
            assert arr.flags['C_CONTIGUOUS']
        self.pixelization = pixelization
        self.nypix_global = pixelization.nypix_global
        self.nxpix_global = pixelization.nxpix_global
        self.periodic_xcoord = pixelization.periodic_xcoord
        self.on_gpu = on_gpu
        self.npix = pixelization.npix
        self.dtype = np.float32
        self.arr = arr

    def to_global(self, on_device=False):
        """The map as a numpy array of shape (3, nypix_global, nxpix_global); pixels outside the
        local map are zero (gpu_mm.py:565-580).  on_device=True (GPU maps): a CUDA tensor, built by a
        kernel without a round trip through the host."""
        if on_device:
            if not (isinstance(self.arr, torch.Tensor) and self.arr.is_cuda):
                raise RuntimeError("LocalMap.to_global(on_device=True): the map is not on the GPU")
            dst = torch.empty((3, self.nypix_global, self.nxpix_global), dtype=torch.float32, device="cuda")
            gpu_mm_pybind11.local_map_to_global(self.pixelization, dst, self.arr)
            return dst
        src = self.arr.detach().cpu().numpy() if isinstance(self.arr, torch.Tensor) else self.arr
        src = np.ascontiguousarray(src.reshape(-1))
        dst = np.zeros((3, self.nypix_global, self.nxpix_global), dtype=np.float32)
        gpu_mm_pybind11.local_map_to_global(self.pixelization, dst, src)
        return dst


####################################################################################################


class DynamicMap:
    """
    A local map that grows while tod2map() runs (the reference's DynamicMap, gpu_mm.py:586-806, with
    the same constructor, methods and errors).  It starts with no cells; every tod2map() into it,
    which needs a PointingPlan, first adds the cells that plan touches, zero-filled, then accumulates.
    finalize() ends the growth and returns a LocalMap.  map2tod() does not take a DynamicMap.

    Storage: float32 [ncells][3][64][64] on the device, cells in the order they were first touched
    (unspecified between runs), or in the order given to permute().  The cell table is the device
    cell_offsets array of a LocalPixelization: -1 marks a cell that may still be added, -2 a cell
    outside 'cell_mask' (bool (nycells, nxcells), True where cells may be added), offsets >= 0 the
    cells present.  New cells are found and numbered on the device (expand_dynamic_map2); only their
    number comes back to the host.  The cell buffer is a capacity of whole cells that grows to the
    next power of two when it overflows (one device copy per growth), so N cells cost O(log N)
    reallocations.
    """

    _GROWING, _PERMUTED, _FINALIZED = 0, 1, 2
    _CELL = 3 * 64 * 64

    def __init__(self, nypix_global, nxpix_global, dtype, cell_mask=None, periodic_xcoord=True, initial_ncells=1024):
        assert 0 < nypix_global <= 64 * 1024
        assert 0 < nxpix_global <= 64 * 1024
        assert np.dtype(dtype) == np.float32 or dtype == torch.float32, "DynamicMap: only float32 maps"
        assert initial_ncells > 0
        self.nypix_global, self.nxpix_global = nypix_global, nxpix_global
        self.periodic_xcoord = periodic_xcoord
        self.dtype = np.float32
        self.have_cell_mask = cell_mask is not None
        shape = ((nypix_global + 63) // 64, (nxpix_global + 63) // 64)
        if cell_mask is None:
            table = np.full(shape, -1, dtype=np.int64)
        else:
            cell_mask = np.asarray(cell_mask)
            assert cell_mask.ndim == 2 and cell_mask.dtype == bool, "DynamicMap: cell_mask must be a 2-d bool array"
            table = np.where(cell_mask, -1, -2).astype(np.int64)
        # The cell layout [ncells][3][64][64]: ystride 64, polstride 64*64.
        self._unstable_pixelization = LocalPixelization(nypix_global, nxpix_global, table, ystride=64,
                                                        polstride=64 * 64, periodic_xcoord=periodic_xcoord)
        self.global_ncells = torch.zeros(32, dtype=torch.int32, device="cuda")[:1]   # device cell counter
        self._cells = torch.zeros((initial_ncells, 3, 64, 64), dtype=torch.float32, device="cuda")
        self._n = 0
        self._state = self._GROWING
        self._view()

    # Read-only state under the reference's attribute names.
    ncells_curr = property(lambda self: self._n)
    ncells_allocated = property(lambda self: self._n if self._cells is None else int(self._cells.shape[0]))
    pixelization_is_finalized = property(lambda self: self._state != self._GROWING)
    map_is_finalized = property(lambda self: self._state == self._FINALIZED)

    def _view(self):
        """Points the pixelization's npix and the flat map array at the cells present."""
        self._unstable_pixelization.npix = 64 * 64 * self._n
        self._unstable_arr = self._cells[:self._n].view(-1)

    def _reserve(self, n):
        cap = int(self._cells.shape[0])
        if n <= cap:
            return
        grown = torch.zeros((1 << (n - 1).bit_length(), 3, 64, 64), dtype=torch.float32, device="cuda")
        grown[:self._n].copy_(self._cells[:self._n])
        self._cells = grown

    def expand(self, plan):
        """Adds the cells 'plan' touches (zero-filled), as tod2map() does before accumulating."""
        if self._state != self._GROWING:
            raise RuntimeError("Can't currently call tod2map() [or DynamicMap.expand()]"
                               + " after MpiPixelization.__init__() [or DynamicMap.permute()].")
        assert isinstance(plan, PointingPlan)
        assert (plan.nypix_global, plan.nxpix_global) == (self.nypix_global, self.nxpix_global)
        assert plan.periodic_xcoord == self.periodic_xcoord
        n = gpu_mm_pybind11.expand_dynamic_map2(self.global_ncells, self._unstable_pixelization, plan)
        self._reserve(n)
        self._n = n
        self._view()

    def permute(self, iycells, ixcells):
        """Puts the cells in the order (iycells[i], ixcells[i]), i = 0..ncells-1 (host integer arrays
        naming every present cell once), and ends the growth of the pixelization.  The data move is
        one gather of whole cells on the device (cell_broadcast)."""
        if self._state != self._GROWING:
            raise RuntimeError("Can't currently call MpiPixelization.__init__() [or DynamicMap.permute()]"
                               + " after DynamicMap.finalize() [or MpiPixelization.__init__(), DynamicMap.permute()]")
        lp = self._unstable_pixelization
        lp.copy_gpu_offsets_to_cpu()
        table = lp.cell_offsets_cpu
        n = self._n
        assert isinstance(iycells, np.ndarray) and isinstance(ixcells, np.ndarray), "permute(): host arrays"
        assert iycells.shape == ixcells.shape == (n,)
        assert np.issubdtype(iycells.dtype, np.integer) and np.issubdtype(ixcells.dtype, np.integer)
        if n:
            assert 0 <= iycells.min() and iycells.max() < table.shape[0]
            assert 0 <= ixcells.min() and ixcells.max() < table.shape[1]
        flat = iycells.astype(np.int64) * table.shape[1] + ixcells.astype(np.int64)
        if not np.array_equal(np.sort(flat), np.flatnonzero(table >= 0)):
            raise RuntimeError('DynamicMap.permute(): specified (iycells,ixcells) do not match footprint of current pixelization')
        src = table[iycells, ixcells] // self._CELL          # current position of each new cell
        table[iycells, ixcells] = self._CELL * np.arange(n, dtype=np.int64)
        lp.copy_cpu_offsets_to_gpu()
        out = torch.empty((n, 3, 64, 64), dtype=torch.float32, device="cuda")
        if n:
            gpu_mm_pybind11.cell_broadcast(out.view(-1), self._cells[:n].reshape(-1),
                                           torch.as_tensor(src, dtype=torch.int64, device="cuda"))
        self._cells = out
        self._state = self._PERMUTED
        self._view()

    def finalize(self):
        """Ends the TOD loop: returns the LocalMap (its pixelization lists the cells present, with
        cell_offsets[iycell, ixcell] = 3*64*64 * i for the i-th cell; absent cells are negative)."""
        if self._state == self._FINALIZED:
            raise RuntimeError('Double call to DynamicMap.finalize() [not currently allowed]')
        if self._state == self._GROWING:
            self._unstable_pixelization.copy_gpu_offsets_to_cpu()
        cells = self._cells[:self._n]
        if self._cells.shape[0] > self._n:
            cells = cells.clone()                 # drop the spare capacity
        ret = LocalMap(self._unstable_pixelization, cells.view(-1))
        assert self._unstable_pixelization.npix == 64 * 64 * self._n
        self._cells = self._unstable_arr = None
        self._state = self._FINALIZED
        return ret

    def randomly_permute(self):
        """permute() into a random order of the present cells (for tests of permute())."""
        self._unstable_pixelization.copy_gpu_offsets_to_cpu()
        iy, ix = np.nonzero(self._unstable_pixelization.cell_offsets_cpu >= 0)
        order = np.random.permutation(len(iy))
        self.permute(iy[order], ix[order])


####################################################################################################


class PointingPrePlan(gpu_mm_pybind11.PointingPrePlan):
    """
    First step of plan construction (gpu_mm.py:1208-1259): counts (cell, cache line) pairs per
    planner block and sizes the PointingPlan buffers.  Small (a few KB); keep one per TOD.

    Constructor: PointingPrePlan(xpointing_gpu, nypix_global, nxpix_global, buf=None, tmp_buf=None,
    periodic_xcoord=True, debug=False).  'buf' and 'tmp_buf' are 1-d 32-bit device arrays of length
    PointingPrePlan.preplan_size; the preplan keeps 'buf' (it holds nmt_cumsum), 'tmp_buf' may be shared.

    Members (from C++): nsamp, nypix_global, nxpix_global, periodic_xcoord, plan_nbytes,
    plan_constructor_tmp_nbytes, overhead, ncl_per_threadblock, planner_nblocks,
    nmt_per_threadblock, pointing_nblocks, plan_nmt, cub_nbytes, get_nmt_cumsum().
    """

    preplan_size = gpu_mm_pybind11.PointingPrePlan._get_preplan_size()

    def __init__(self, xpointing_gpu, nypix_global, nxpix_global, buf=None, tmp_buf=None, periodic_xcoord=True, debug=False):
        if buf is None:
            buf = torch.empty(self.preplan_size, dtype=torch.int32, device="cuda")
        if tmp_buf is None:
            tmp_buf = torch.empty(self.preplan_size, dtype=torch.int32, device="cuda")
        self._buf = buf
        gpu_mm_pybind11.PointingPrePlan.__init__(self, xpointing_gpu, nypix_global, nxpix_global, buf, tmp_buf,
                                                 periodic_xcoord, debug)


class PointingPlan(gpu_mm_pybind11.PointingPlan):
    """
    The plan argument of map2tod()/tod2map() (gpu_mm.py:1262-1299): mt words sorted by
    (cell, cache line) -- the reference's plan_mt, reproduced bit for bit in canonical order -- plus
    one owner word per cache line, which the operators use to visit every line once.

    Constructor: PointingPlan(preplan, xpointing_gpu, buf=None, tmp_buf=None, debug=False).  'buf'
    (uint8, >= preplan.plan_nbytes) is kept by the plan; 'tmp_buf' (uint8, >=
    preplan.plan_constructor_tmp_nbytes) is only used during construction and may be shared.
    """

    def __init__(self, preplan, xpointing_gpu, buf=None, tmp_buf=None, debug=False):
        if buf is None:
            buf = torch.empty(preplan.plan_nbytes, dtype=torch.uint8, device="cuda")
        if tmp_buf is None:
            tmp_buf = torch.empty(preplan.plan_constructor_tmp_nbytes, dtype=torch.uint8, device="cuda")
        self._buf = buf
        self.preplan = preplan
        gpu_mm_pybind11.PointingPlan.__init__(self, preplan, xpointing_gpu, buf, tmp_buf, debug)


class ToyPointing(gpu_mm_pybind11.ToyPointing):
    """
    ToyPointing(ndet, nt, nypix_global, nxpix_global, scan_speed, total_drift, noisy=True)
    (gpu_mm.py:1332-1385): a synthetic raster for tests.  Scans go at 45 degrees and cover the
    full y range; 'scan_speed' = map pixels per TOD sample, 'total_drift' = drift over the TOD in
    x-pixels.  ndet=None gives (3, nt) pointing, else (3, ndet, nt).

    Members: xpointing_cpu (numpy float32), xpointing_gpu (torch CUDA float32), ndet, nt, and from
    C++ nypix_global, nxpix_global, scan_speed, total_drift, drift_speed, __str__().
    """

    def __init__(self, ndet, nt, nypix_global, nxpix_global, scan_speed, total_drift, noisy=True):
        shape = (3, ndet, nt) if (ndet is not None) else (3, nt)
        self.ndet, self.nt = ndet, nt
        self.xpointing_cpu = np.zeros(shape, mm_dtype)
        self.xpointing_gpu = torch.zeros(shape, dtype=torch.float32, device="cuda")
        gpu_mm_pybind11.ToyPointing.__init__(self, nypix_global, nxpix_global, scan_speed, total_drift,
                                             self.xpointing_cpu, self.xpointing_gpu, noisy)

    @staticmethod
    def make_random(nsamp_max, noisy=True):
        """A ToyPointing of random shape and parameters (the reference's make_random): TOD shape (nt,)
        or (ndet, nt) with at most about nsamp_max samples."""
        assert nsamp_max >= 64 * 1024
        if np.random.randint(0, 2):
            ndet = None
            nt = 32 * np.random.randint(nsamp_max // 64, nsamp_max // 32)
        else:
            r = np.random.randint(0, 6)
            s = int((nsamp_max / 32.) ** 0.5)
            ndet = 2 ** r * np.random.randint(s // 2, s + 1)
            nt = 2 ** (5 - r) * np.random.randint(s // 2, s + 1)
        npix_max = min(nsamp_max // 128, 16384)
        nypix_global = np.random.randint(npix_max / 8, npix_max // 2 + 1)
        nxpix_global = np.random.randint(nypix_global + 2, npix_max + 1)
        scan_speed = np.random.uniform(0.1, 0.5)
        total_drift = np.random.uniform(0.1 * (nxpix_global - nypix_global), (nxpix_global - nypix_global) - 2)
        return ToyPointing(ndet, nt, nypix_global, nxpix_global, scan_speed, total_drift, noisy=noisy)


class PointingPlanTester(gpu_mm_pybind11.PointingPlanTester):
    """
    PointingPlanTester(preplan, xpointing_gpu) (gpu_mm.py:1388-1415): the plan computed the simple way,
    for tests.  Members: nsamp, nypix_global, nxpix_global, plan_nmt, ncl_per_threadblock,
    planner_nblocks, iypix and ixpix (per sample, from the GPU), nmt_cumsum (per planner block) and
    sorted_mt (all mt words, sorted), as numpy arrays.
    """

    def __init__(self, preplan, xpointing_gpu):
        assert isinstance(preplan, PointingPrePlan)
        tmp_nbytes = gpu_mm_pybind11.PointingPlanTester.get_constructor_tmp_nbytes(preplan)
        tmp = torch.empty(tmp_nbytes, dtype=torch.uint8, device="cuda")
        gpu_mm_pybind11.PointingPlanTester.__init__(self, preplan, xpointing_gpu, tmp)


####################################################################################################


def read_xpointing_npzfile(filename):
    """Reads a (3, ndet, nt) xpointing array from the reference's ad hoc .npz format
    (gpu_mm.py:1305-1329): rows stored as (x, y, alpha), nt padded to a multiple of 32."""
    f = np.load(filename)
    xp = f['xpointing']
    assert (xp.ndim == 3) and (xp.shape[0] == 3)
    ndet = xp.shape[1]
    ntu = xp.shape[2]
    ntp = 32 * ((ntu + 31) // 32)
    xpointing_cpu = np.zeros((3, ndet, ntp), dtype=xp.dtype)
    xpointing_cpu[0, :, :ntu] = xp[1, :, :]
    xpointing_cpu[1, :, :ntu] = xp[0, :, :]
    xpointing_cpu[2, :, :ntu] = xp[2, :, :]
    xpointing_cpu[:, :, ntu:] = xpointing_cpu[:, :, ntu - 1].reshape((3, -1, 1))
    return xpointing_cpu
