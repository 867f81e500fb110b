/*
 * gpu_mm_b200: C ABI of the B200-native pointing-operator hot path.
 *
 * This is the drop-in boundary.  Every entry point replaces one piece of the reference's C++
 * interface (kmsmith137/gpu_mm, include/gpu_mm.hpp); the comment above each one names it.  The
 * signatures use plain pointers, 64-bit sizes and a cudaStream_t, and no C++ or torch types.  The
 * C++ API (include/gpu_mm_b200/gpu_mm.hpp) and the pybind11 module gpu_mm_pybind11 sit on top.
 *
 * Conventions
 *  - Device arrays are raw device pointers, float32 (the reference's pybind layer wraps float32
 *    only, gpu_mm_pybind11.cu:17-19).  TODs are flat [nsamp]; xpointing is [3][nsamp] with rows
 *    {y, x, alpha} (gpu_mm.py:59-85).
 *  - Every function returns an int status.  0 means success.  Values 1, 2, 4 and 8 are the reference's
 *    device error bits (gpu_mm_internals.hpp:26-29); GMM_ERR_* >= 0x100 are API errors.  The last
 *    error message of the calling thread is available from gmm_last_error().
 *  - The device error bits of an operator call are OR-reduced on the device into one 32-bit word.
 *    If 'errword_gpu' is NULL, the call reads that word back on 'stream' and returns its bits, which
 *    is synchronous like the reference (check_arguments.cu:69-74).  Otherwise the word is left on
 *    the device for a deferred check with gmm_errword_read(), and the call does not block.
 *  - No function allocates device memory.  Callers own every buffer, as with the reference's Python
 *    constructors (gpu_mm.py:1253-1259, :1293-1299).
 */
#ifndef GPU_MM_B200_H
#define GPU_MM_B200_H

#include <stdint.h>
#include <cuda_runtime_api.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GMM_ERR_BAD_YPIX 0x1
#define GMM_ERR_BAD_XPIX 0x2
#define GMM_ERR_INCONSISTENT_NMT 0x4
#define GMM_ERR_NOT_IN_PIXELIZATION 0x8
#define GMM_ERR_INVALID_ARGUMENT 0x100
#define GMM_ERR_CUDA 0x200
#define GMM_ERR_BUFFER_TOO_SMALL 0x400

/* Size of the nmt/err buffers owned by a preplan (gpu_mm.hpp:63, PointingPrePlan::preplan_size). */
#define GMM_PREPLAN_SIZE 1024

/* Local pixelization as seen by the device: LocalPixelization (gpu_mm.hpp:17-58). */
typedef struct gmm_lpix {
    int32_t nypix_global;
    int32_t nxpix_global;
    int32_t periodic_xcoord;
    int32_t nycells;              /* cell_offsets.shape[0], <= 1024 */
    int32_t nxcells;              /* cell_offsets.shape[1], <= 1024 */
    int32_t reserved;
    int64_t ystride;
    int64_t polstride;
    int64_t npix;                 /* local pixels (map size is 3*npix) */
    const int64_t *cell_offsets;  /* device pointer, [nycells][nxcells], negative = absent */
} gmm_lpix;

/* Scalars of a PointingPrePlan (gpu_mm.hpp:79-101, PointingPrePlan.cu:159-250).  The launch
 * geometry fields (ncl_per_threadblock .. pointing_nblocks, plan_nmt) equal the reference's;
 * plan_nbytes / plan_constructor_tmp_nbytes are this implementation's buffer sizes. */
typedef struct gmm_preplan_info {
    int64_t nsamp;
    int32_t nypix_global;
    int32_t nxpix_global;
    int32_t periodic_xcoord;
    int32_t sort_digit_bits;      /* radix digit width chosen for the plan sort */
    int64_t plan_nbytes;
    int64_t plan_constructor_tmp_nbytes;
    double overhead;
    int64_t ncl_per_threadblock;
    int64_t planner_nblocks;
    int64_t nmt_per_threadblock;
    int64_t pointing_nblocks;
    int64_t plan_nmt;
    int64_t sort_nbytes;          /* replaces PointingPrePlan::cub_nbytes: scratch of the radix sort */
} gmm_preplan_info;

/* Byte offsets of the arrays inside a plan buffer (the reference's 'buf' holds plan_mt and err,
 * PointingPlan.cu:251-260; this layout appends the owner-line list, the cell bitmap and the band
 * words of the tod2map band path). */
typedef struct gmm_plan_layout {
    int64_t mt_offset;        /* uint64 plan_mt[plan_nmt], sorted by (cell, cache line) */
    int64_t err_offset;       /* uint32 err[max(planner_nblocks, pointing_nblocks)] */
    int64_t owner_offset;     /* uint64 owner_mt[nsamp/32]: one word per cache line, sorted */
    int64_t cellmap_offset;   /* uint32 cellmap[2^20/32]: bit c set iff cell c occurs in plan_mt */
    int64_t total_nbytes;
    int64_t band_offset;      /* uint64 band[nsamp/32]: per owner entry, the line's shape for tod2map */
} gmm_plan_layout;

/* Thread-local message of the last failing call on this thread ("" if none). */
const char *gmm_last_error(void);

/* Library version string. */
const char *gmm_version(void);

/* Maximum radix digit width (4..11 bits) of the plan sort, used by later gmm_preplan calls.  The
 * reference's sort is CUB's (PointingPlan.cu:300-309), whose digit width is not a parameter; here
 * it is a tuning knob set by the autotuner (gpu_mm_b200/autotune.py).  Default 8. */
int gmm_set_sort_digit_bits(int32_t bits);
int gmm_get_sort_digit_bits(void);

/* Kernel of the plain (float) planned tod2map of single-TOD plans, for later calls in this process.
 * The reference has one tod2map kernel (tod2map.cu:16-150: shared-memory tile per cell, one
 * atomic per sample and pixel); here there are two, which give the same result within float
 * rounding:
 *   GMM_TOD2MAP_BANDS (default): lines grouped by (cell, row band) in the plan; each warp sums a
 *     band's lines in its own shared-memory accumulator and adds them to the map once per band
 *     (every flush mode);
 *   GMM_TOD2MAP_TILES: shared-memory tile of each cell plus halo, as batches use (and single-TOD
 *     calls whose xpointing or TOD is not 16-byte aligned).
 * A tuning knob: the bands kernel is faster for raster scans, the tiles kernel for pointing that
 * is not (e.g. scans faster than one pixel per sample or rotated against the pixel grid). */
#define GMM_TOD2MAP_BANDS 0
#define GMM_TOD2MAP_TILES 1
int gmm_set_planned_tod2map_kernel(int32_t which);
int gmm_get_planned_tod2map_kernel(void);

/* Replaces the PointingPrePlan constructor (PointingPrePlan.cu:129-251 / gpu_mm.hpp:74-77).
 * Counts mt words per planner block on the device, writes the inclusive cumsum (padded with the
 * total) to nmt_gpu[GMM_PREPLAN_SIZE], uses err_gpu[GMM_PREPLAN_SIZE] as scratch, and fills *info.
 * Synchronises with 'stream' once (to learn nmt), like the reference constructor. */
int gmm_preplan(const float *xpointing_gpu, int64_t nsamp, int32_t nypix_global, int32_t nxpix_global,
                int32_t periodic_xcoord, uint32_t *nmt_gpu, uint32_t *err_gpu, int32_t debug,
                cudaStream_t stream, gmm_preplan_info *info);

/* Computes the host-side PointingPrePlan scalars from nsamp and nmt (no device work). */
int gmm_preplan_info_init(int64_t nsamp, int32_t nypix_global, int32_t nxpix_global, int32_t periodic_xcoord,
                          int64_t nmt, gmm_preplan_info *info);

/* Layout of a plan buffer for a given preplan. */
int gmm_plan_layout_get(const gmm_preplan_info *info, gmm_plan_layout *layout);

/* Replaces the PointingPlan constructor (PointingPlan.cu:237-312 / gpu_mm.hpp:132-137): emits the
 * mt words, sorts them with the hand-written radix sort and builds the owner-line list.
 * 'buf' needs info->plan_nbytes bytes and 'tmp' info->plan_constructor_tmp_nbytes bytes, both
 * 128-byte aligned device memory.  Synchronises once to check the error flags (PointingPlan.cu:311). */
int gmm_plan_build(const gmm_preplan_info *info, const uint32_t *nmt_cumsum_gpu, const float *xpointing_gpu,
                   void *buf, int64_t buf_nbytes, void *tmp, int64_t tmp_nbytes, int32_t debug,
                   cudaStream_t stream);

/* Plan construction for callers that cannot allocate device memory.  This entry point has no
 * counterpart in the reference.  It is gmm_plan_build without the 'tmp' argument: its temporary
 * storage (the unsorted mt words, the second owner-list buffer and the radix-sort histograms) lives
 * in a static device array of GMM_NOALLOC_SCRATCH_BYTES (32 MiB) inside this library.  It is meant
 * for hosts that must not call cudaMalloc -- real-time acquisition loops, code that hands out device
 * memory from its own fixed pool, foreign-language runtimes without a device allocator -- and that
 * still need to build plans.  The caller passes the inputs (preplan, nmt_cumsum, xpointing) and the
 * output 'buf' as usual.
 *  - Plans whose info->plan_constructor_tmp_nbytes exceeds GMM_NOALLOC_SCRATCH_BYTES are rejected
 *    with GMM_ERR_BUFFER_TOO_SMALL; that covers up to roughly 2^24 samples at typical overheads.
 *  - The array is reserved on every device where this library's module holding it has been loaded
 *    and is kept until the process exits.
 *  - The first call on a device looks up the array's device address (cudaGetSymbolAddress).
 *  - All calls share the one array.  Calls that overlap on the GPU (other streams, other host
 *    threads) race on it and must be serialised by the caller.  Nothing in the array needs to
 *    start at zero: every call overwrites what it reads.
 *  - Like gmm_plan_build, each call synchronises with 'stream' once, to read the error flags.
 * Allocates nothing. */
#define GMM_NOALLOC_SCRATCH_BYTES (32ll << 20)
int gmm_plan_build_noalloc(const gmm_preplan_info *info, const uint32_t *nmt_cumsum_gpu, const float *xpointing_gpu,
                           void *buf, int64_t buf_nbytes, int32_t debug, cudaStream_t stream);

/* Replaces launch_planned_map2tod<float> (gpu_mm.hpp:155-165, map2tod.cu:194-272). */
int gmm_planned_map2tod(float *tod, const float *local_map, const float *xpointing, const gmm_lpix *lpix,
                        const gmm_preplan_info *info, const void *plan_buf, int32_t partial_pixelization,
                        int32_t accum, uint32_t *errword_gpu, cudaStream_t stream);

/* Replaces launch_planned_tod2map<float> (gpu_mm.hpp:168-177, tod2map.cu:157-226).  Accumulates. */
int gmm_planned_tod2map(float *local_map, const float *tod, const float *xpointing, const gmm_lpix *lpix,
                        const gmm_preplan_info *info, const void *plan_buf, int32_t partial_pixelization,
                        uint32_t *errword_gpu, cudaStream_t stream);

/* Replaces local_map_to_global (gpu_mm.hpp:226-228, local_map_to_global.cu:12-44) for device arrays:
 * dst is the dense (3, nypix_global, nxpix_global) global map (zeroed outside the local cells). */
int gmm_local_map_to_global(float *dst, const float *src, const gmm_lpix *lpix, cudaStream_t stream);

/* Replace cell_broadcast / cell_reduce (gpu_mm.hpp:230-236, cell_broadcast.cu, cell_reduce.cu) for
 * device arrays of cell-major buffers (3*64*64 floats per cell): broadcast dst cell i = src cell
 * index_map[i]; reduce dst = 0, then dst cell index_map[i] += src cell i.  index_map is a device
 * int64 array of ncells entries; out-of-range entries are skipped and set bit 1 of the error word. */
int gmm_cell_broadcast(float *dst, const float *src, int64_t nsrc, const int64_t *index_map_gpu, int64_t ncells,
                       uint32_t *errword_gpu, cudaStream_t stream);
int gmm_cell_reduce(float *dst, int64_t ndst, const float *src, const int64_t *index_map_gpu, int64_t ncells,
                    uint32_t *errword_gpu, cudaStream_t stream);

/* ---- TOD preprocessing (the reference's deglitching.cu, cuts.cu, misc.cu), device arrays.
 * Every index read from an index map is checked against the arrays' extents; entries out of range
 * are skipped and set bit 1 of the error word (zeroed by each call). */

/* get_border_means (deglitching.cu:99-141): out[r] = (mean signal[di, b00:b01], mean signal[di, b10:b11])
 * for index_map[r] = (di, b00, b01, b10, b11); an empty range takes the other's mean.  signal is
 * (ndet, nt), out (R, 2), index_map (R, 5) int32. */
int gmm_get_border_means(float *out, const float *signal, int64_t ndet, int64_t nt, const int32_t *index_map,
                         int64_t R, uint32_t *errword_gpu, cudaStream_t stream);

/* deglitch (deglitching.cu:180-210, gpu_mm.py:1461-1501): cumj = cumsum(bvals[:,1] - bvals[:,0]) into
 * the caller's scratch 'cumj' (R floats), then per range r = (di, r0, t1, t2) of index_map2 (R, 4):
 * signal[di, t1:t2] = bvals[r,1] - dc and signal[di, t2:t3] -= dc, with dc = cumj[r] - cumj[r0-1]. */
int gmm_deglitch(float *signal, int64_t ndet, int64_t nt, const float *bvals, const int32_t *index_map2, int64_t R,
                 float *cumj, uint32_t *errword_gpu, cudaStream_t stream);
/* deglitch with the jump cumsum given by the caller (the reference's pybind deglitch(signal, bvals,
   cumj, index_map2), deglitching.cu:180-210): cumj (R,) float32 on the device. */
int gmm_deglitch_cumj(float *signal, int64_t ndet, int64_t nt, const float *bvals, const float *cumj,
                      const int32_t *index_map2, int64_t R, uint32_t *errword, cudaStream_t stream);

/* extract_ranges / insert_ranges / clear_ranges (cuts.cu:38-55): range r is
 * tod[det[r], istart[r] : istart[r] + len[r]] of a (ndet, nsamp) TOD, kept in rdata[ostart[r]:]. */
int gmm_extract_ranges(const float *tod, int64_t ndet, int64_t nsamp, float *rdata, int64_t nrdata,
                       const int32_t *ostart, const int32_t *det, const int32_t *istart, const int32_t *len,
                       int64_t nrange, uint32_t *errword_gpu, cudaStream_t stream);
int gmm_insert_ranges(float *tod, int64_t ndet, int64_t nsamp, const float *rdata, int64_t nrdata,
                      const int32_t *ostart, const int32_t *det, const int32_t *istart, const int32_t *len,
                      int64_t nrange, uint32_t *errword_gpu, cudaStream_t stream);
int gmm_clear_ranges(float *tod, int64_t ndet, int64_t nsamp, const int32_t *det, const int32_t *istart,
                     const int32_t *len, int64_t nrange, uint32_t *errword_gpu, cudaStream_t stream);

/* clip (misc.cu:8-19): arr = max(vmin, min(vmax, arr)) in place. */
int gmm_clip(float *arr, int64_t n, float vmin, float vmax, cudaStream_t stream);

/* ---- Batches of TODs (no counterpart in the reference, which plans and applies one TOD per call).
 *
 * A batch is up to 65535 TODs, each with its own xpointing [3][nsamp] and TOD [nsamp] (16-byte
 * aligned, nsamp a positive multiple of 32), against one local pixelization.  The caller keeps an
 * array of gmm_tod_desc in device memory; line0 of TOD i is the sum of nsamp/32 over TODs < i, and
 * total_lines the sum over all.  A batch plan is one owner list over all the batch's cache lines,
 * sorted by cell (tile loads are shared by every TOD that hits a cell), plus the bitmap of cells the
 * lines touch.  Its size depends only on total_lines, so building it needs no host synchronisation
 * and can be captured in a CUDA graph together with the operators.  Device error bits go to
 * 'errword_gpu' (required; read it with gmm_errword_read). */
typedef struct gmm_tod_desc {
    const float *xpointing;   /* [3][nsamp] */
    float *tod;               /* [nsamp]: map2tod output, tod2map input */
    int64_t nsamp;
    int64_t line0;
} gmm_tod_desc;

/* Launch and sort parameters of the batched kernels (gmm_batch_tuning_default fills the defaults;
 * an autotuner may pick others).  sort_digit_bits: radix digit width of the plan sort (4..11);
 * ctas_per_sm: operator CTAs per SM in the grid (1..8, two are resident at a time);
 * min_lines_per_cta: lower bound on the cache lines of one CTA's slice. */
typedef struct gmm_batch_tuning {
    int32_t sort_digit_bits;
    int32_t ctas_per_sm;
    int32_t min_lines_per_cta;
    int32_t reserved;
} gmm_batch_tuning;

int gmm_batch_tuning_default(gmm_batch_tuning *tuning);

/* Sizes of a batch plan and of its construction scratch. */
int gmm_batch_plan_nbytes(int64_t total_lines, int32_t nypix_global, int32_t nxpix_global,
                          const gmm_batch_tuning *tuning, int64_t *plan_nbytes, int64_t *tmp_nbytes);

/* Builds the batch plan into 'plan_buf' (128-byte aligned) using 'tmp' (128-byte aligned). */
int gmm_batch_plan_build(const gmm_tod_desc *descs_gpu, int32_t ntod, int64_t total_lines, int32_t nypix_global,
                         int32_t nxpix_global, int32_t periodic_xcoord, void *plan_buf, int64_t plan_nbytes, void *tmp,
                         int64_t tmp_nbytes, const gmm_batch_tuning *tuning, uint32_t *errword_gpu, cudaStream_t stream);

/* Builds the single-TOD plans of up to 4096 TODs at once: plans_gpu[i] (device array of ntod
 * pointers) receives TOD i's plan, laid out as gmm_batch_plan_build with ntod = 1 lays it out (sized
 * by gmm_batch_plan_nbytes(nsamp_i/32, ...), 128-byte aligned).  One owner pass over all the TODs,
 * one sort by (TOD, cell), one scatter; 'tmp' sized by gmm_batch_plan_each_tmp_nbytes. */
int gmm_batch_plan_each_tmp_nbytes(int64_t total_lines, int32_t ntod, int32_t nypix_global, int32_t nxpix_global,
                                   const gmm_batch_tuning *tuning, int64_t *tmp_nbytes);
int gmm_batch_plan_build_each(const gmm_tod_desc *descs_gpu, int32_t ntod, int64_t total_lines, int32_t nypix_global,
                              int32_t nxpix_global, int32_t periodic_xcoord, void *const *plans_gpu, void *tmp,
                              int64_t tmp_nbytes, const gmm_batch_tuning *tuning, uint32_t *errword_gpu,
                              cudaStream_t stream);

/* Merges single-TOD batch plans (each built by gmm_batch_plan_build with ntod = 1) into the plan of
 * a batch whose TOD i has plans_gpu[i]: the owner words are copied with their TOD index set to i,
 * the cell bitmaps OR-ed, and the list sorted by cell (stable: the order gmm_batch_plan_build gives
 * for the same batch).  plans_gpu and nlines_gpu are device arrays of ntod entries; nlines[i] is TOD
 * i's line count (its nsamp/32); their sum is total_lines.  'plan_buf' and 'tmp' are sized by
 * gmm_batch_plan_nbytes(total_lines, ...). */
int gmm_batch_plan_merge(const void *const *plans_gpu, const int64_t *nlines_gpu, int32_t ntod, int64_t total_lines,
                         int32_t nypix_global, int32_t nxpix_global, void *plan_buf, int64_t plan_nbytes, void *tmp,
                         int64_t tmp_nbytes, const gmm_batch_tuning *tuning, cudaStream_t stream);

/* map2tod / tod2map of every TOD of the batch in one launch each, with the semantics of
 * gmm_planned_map2tod / gmm_planned_tod2map per TOD. */
int gmm_batch_map2tod(const gmm_tod_desc *descs_gpu, int32_t ntod, int64_t total_lines, const float *local_map,
                      const gmm_lpix *lpix, const void *plan_buf, int32_t partial_pixelization, int32_t accum,
                      const gmm_batch_tuning *tuning, uint32_t *errword_gpu, cudaStream_t stream);
int gmm_batch_tod2map(const gmm_tod_desc *descs_gpu, int32_t ntod, int64_t total_lines, float *local_map,
                      const gmm_lpix *lpix, const void *plan_buf, int32_t partial_pixelization,
                      const gmm_batch_tuning *tuning, uint32_t *errword_gpu, cudaStream_t stream);

/* Precision variants of planned tod2map.  No counterpart in the reference, whose tod2map
 * accumulates in float only (tod2map.cu:157-226); its sample arithmetic is unchanged here (float
 * arithmetic and partial sums), only the reduction into the map differs:
 *   _compensated: float map plus a float 'comp' array of the same size (caller-owned, zeroed
 *                 before the first call) that collects the rounding error of every float addition
 *                 into the map (two-sum).  local_map + comp then holds the sum to about twice float
 *                 precision; gmm_fold_compensation adds comp into local_map and zeroes comp.
 *   _f64:         double local map (same cell_offsets / ystride / polstride, in doubles); partials
 *                 are reduced with double atomics.
 * max_run_lines > 0 bounds how many cache lines a partial collects before it is reduced into the
 * map (0: at each change of cell, or of cell and row band on the row-band kernel). */
int gmm_planned_tod2map_compensated(float *local_map, float *comp, const float *tod, const float *xpointing,
                                    const gmm_lpix *lpix, const gmm_preplan_info *info, const void *plan_buf,
                                    int32_t partial_pixelization, int64_t max_run_lines, uint32_t *errword_gpu,
                                    cudaStream_t stream);
int gmm_planned_tod2map_f64(double *local_map, const float *tod, const float *xpointing, const gmm_lpix *lpix,
                            const gmm_preplan_info *info, const void *plan_buf, int32_t partial_pixelization,
                            int64_t max_run_lines, uint32_t *errword_gpu, cudaStream_t stream);
int gmm_fold_compensation(float *local_map, float *comp, int64_t n, cudaStream_t stream);

/* float64 only where the hit count is high.  No counterpart in the reference.  A float map whose
 * high-hit ("hot") cells have their partial sums reduced with double atomics into a float64
 * accumulator of their own, [nhot][3][64][64], and rounded into the float map once, by
 * gmm_fold_hot_f64; every other cell's partials go into the float map with float atomics, as in
 * gmm_planned_tod2map.
 *   gmm_plan_cell_lines: adds, per cell of lpix's grid, the number of the plan's cache lines that
 *       touch the cell (its mt words) into lines[nycells * nxcells] (uint32, caller-zeroed); call it
 *       for every plan whose TODs will be accumulated.
 *   gmm_hot_cells: hot_slot[c] = the accumulator slot of cell c = iycell * nxcells + ixcell if the
 *       cell is present in lpix and lines[c] >= min_lines (slots in cell order), else -1;
 *       hot_cells[slot] = c; *nhot (device int32) = the number of hot cells.  hot_slot and
 *       hot_cells hold nycells * nxcells entries.
 *   gmm_planned_tod2map_hot_f64: planned tod2map in that mode ('hot': nhot * 3 * 4096 doubles,
 *       zeroed before the first call).  Runs the row-band kernel whatever
 *       gmm_set_planned_tod2map_kernel chose; tod and xpointing must be 16-byte aligned.
 *       max_run_lines bounds the partials of lines owned by hot cells, as for the other precision
 *       variants; the other cells reduce once per (cell, row band), as gmm_planned_tod2map.
 *   gmm_fold_hot_f64: local_map = float(local_map + hot) over the hot cells, hot = 0.
 * hot_slot and hot_cells must be rebuilt if lpix's cell_offsets change. */
int gmm_plan_cell_lines(const gmm_preplan_info *info, const void *plan_buf, const gmm_lpix *lpix, uint32_t *lines_gpu,
                        cudaStream_t stream);
int gmm_hot_cells(const uint32_t *lines_gpu, const gmm_lpix *lpix, uint32_t min_lines, int32_t *hot_slot_gpu,
                  int32_t *hot_cells_gpu, int32_t *nhot_gpu, cudaStream_t stream);
int gmm_planned_tod2map_hot_f64(float *local_map, double *hot, const int32_t *hot_slot_gpu, const float *tod,
                                const float *xpointing, const gmm_lpix *lpix, const gmm_preplan_info *info,
                                const void *plan_buf, int32_t partial_pixelization, int64_t max_run_lines,
                                uint32_t *errword_gpu, cudaStream_t stream);
int gmm_fold_hot_f64(float *local_map, double *hot, const int32_t *hot_cells_gpu, int64_t nhot, const gmm_lpix *lpix,
                     cudaStream_t stream);

/* Replaces launch_response_map2tod<float> / launch_response_tod2map<float> (gpu_mm.hpp:179-202,
 * map2tod_response.cu:205-290, tod2map_response.cu).  response is [2][ndet] (T, P), ndet divides nsamp. */
int gmm_response_map2tod(float *tod, const float *local_map, const float *xpointing, const float *response,
                         int64_t ndet, const gmm_lpix *lpix, const gmm_preplan_info *info, const void *plan_buf,
                         int32_t partial_pixelization, int32_t accum, uint32_t *errword_gpu, cudaStream_t stream);
int gmm_response_tod2map(float *local_map, const float *tod, const float *xpointing, const float *response,
                         int64_t ndet, const gmm_lpix *lpix, const gmm_preplan_info *info, const void *plan_buf,
                         int32_t partial_pixelization, uint32_t *errword_gpu, cudaStream_t stream);

/* Replaces launch_unplanned_map2tod<float> (gpu_mm.hpp:204-213, map2tod_unplanned.cu:74-127).
 * errflags_gpu has errflags_len >= 1 words (the reference's per-block array); word 0 receives the
 * OR of all device error bits. */
int gmm_unplanned_map2tod(float *tod, const float *local_map, const float *xpointing, int64_t nsamp,
                          const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                          int32_t partial_pixelization, int32_t accum, int32_t sync_check, cudaStream_t stream);

/* Replaces launch_unplanned_tod2map<float> (gpu_mm.hpp:216-224, tod2map_unplanned.cu:68-121). */
int gmm_unplanned_tod2map(float *local_map, const float *tod, const float *xpointing, int64_t nsamp,
                          const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                          int32_t partial_pixelization, int32_t sync_check, cudaStream_t stream);

/* Double-precision unplanned operators: replace launch_unplanned_map2tod<double> and
 * launch_unplanned_tod2map<double> (gpu_mm.hpp:204-224, map2tod_unplanned.cu:130-141,
 * tod2map_unplanned.cu:124-134).  Arguments as in the float entry points, with double arrays. */
int gmm_unplanned_map2tod_f64(double *tod, const double *local_map, const double *xpointing, int64_t nsamp,
                              const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                              int32_t partial_pixelization, int32_t accum, int32_t sync_check, cudaStream_t stream);
int gmm_unplanned_tod2map_f64(double *local_map, const double *tod, const double *xpointing, int64_t nsamp,
                              const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                              int32_t partial_pixelization, int32_t sync_check, cudaStream_t stream);

/* Per-sample pixel quantization for the PointingPlanTester test utility (PointingPlanTester.cu:22-63,
 * quantize_kernel): iypix[s], ixpix[s] = the (iy0, ix0) that locate() gives sample s.  Asynchronous;
 * device error bits (out-of-range pointing) go to *errword. */
int gmm_quantize_pointing(const float *xpointing, int64_t nsamp, int32_t nypix_global, int32_t nxpix_global,
                          int32_t periodic_xcoord, int32_t *iypix, int32_t *ixpix, uint32_t *errword,
                          cudaStream_t stream);

/* Deferred error check: reads the device error word (after 'stream' completes), masks the bits in
 * 'ignore' and returns the rest (check_gpu_errflags, check_arguments.cu:69-74). */
int gmm_errword_read(const uint32_t *errword_gpu, uint32_t ignore, cudaStream_t stream);

/* Replaces expand_dynamic_map (gpu_mm.hpp:268-272, expand_dynamic_map.cu:106-141): cells of the
 * sorted plan whose offset is -1 ("targeted") get offsets (global_ncells + i) * 3*64*64.
 * Returns the updated cell count in *ncells_out (synchronous). */
int gmm_expand_dynamic_map(uint32_t *global_ncells_gpu, int64_t *cell_offsets_gpu, int32_t nycells,
                           int32_t nxcells, const uint64_t *plan_mt_gpu, int64_t nmt, uint32_t *ncells_out,
                           cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* GPU_MM_B200_H */
