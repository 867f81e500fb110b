// Internal declarations shared by the gpu_mm_b200 translation units.
#pragma once

#include <atomic>
#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "gmm_common.cuh"
#include "../../include/gpu_mm_b200.h"

extern "C" int gmm_fail_message(int code, const char *msg);

namespace gmm {

// Number of SMs of the current device (cached per device).
int device_sm_count();
// Turns device error bits into the reference's exception text (check_arguments.cu:42-58) as the
// last-error message and returns the status code (0 if no bit outside 'ignore' is set).
int report_err_bits(uint32_t err, const char *where, uint32_t ignore);

// ---- plan construction (plan_kernels.cu) ----
// Radix sort of plan words by cell (and, with tod_bits > 0, by TOD index above the cell; the owner
// words of single-TOD plans by (cell, row band), kBandBits more key bits, passed as tod_bits here).
int sort_passes(int nycells_max, int nxcells_max, int max_digit_bits, int *digit_bits, int tod_bits = 0);
int64_t sort_scratch_nbytes(int digit_bits, int grid);
int sort_grid_for(int64_t n);
cudaError_t radix_sort_mt(uint64_t *a, uint64_t *b, int64_t n, int nycells_max, int nxcells_max, int digit_bits,
                          int npasses, uint32_t *hist, cudaStream_t stream, int tod_bits = 0, int band_bits = 0);
cudaError_t launch_preplan(const float *xp, int64_t nsamp, int ny, int nx, bool periodic, int64_t nclpb,
                           int nblocks, uint32_t *nmt, uint32_t *err, cudaStream_t stream);
cudaError_t launch_plan_emit(const float *xp, int64_t nsamp, int ny, int nx, bool periodic, int64_t nclpb,
                             int nblocks, const uint32_t *nmt_cumsum, uint64_t *mt_out, uint64_t *owner_out,
                             uint64_t *band_out, uint32_t *errflags, cudaStream_t stream);
// Band words (gmm_common.cuh) from line order into owner-list order.
cudaError_t launch_band_gather(const uint64_t *owner, int64_t n, const uint64_t *band_by_line, uint64_t *band_out,
                               cudaStream_t stream);
cudaError_t launch_plan_cellmap(const uint64_t *plan_mt, int64_t nmt, uint32_t *cellmap, cudaStream_t stream);
cudaError_t launch_expand_dynamic_map(uint32_t *global_ncells, int64_t *cell_offsets, int nycells, int nxcells,
                                      const uint64_t *plan_mt, int64_t nmt, cudaStream_t stream);

// ---- operators (operator_kernels.cu) ----
struct OpArgs {
    float *out;             // tod (map2tod) or local map (tod2map)
    const float *in;        // local map (map2tod) or tod (tod2map)
    const float *xp;        // xpointing [3][nsamp]
    const float *response;  // [2][ndet] or nullptr
    int64_t ndet, nperdet;
    // sample -> detector index as a multiply-high (Granlund & Montgomery, "Division by invariant
    // integers using multiplication", PLDI 1994): det = (t + ((s - t) >> sh1)) >> sh2, t = umulhi(m, s).
    uint32_t det_m;
    int det_sh1, det_sh2;
    const int64_t *cell_offsets;
    int64_t nsamp;
    int ny, nx;
    bool periodic;
    int nycells, nxcells;
    int64_t ystride, polstride;
    bool partial, accum;
    uint32_t *errword;
    // tod2map precision modes (planned operators only).  flush: how tile partials and out-of-tile
    // samples reach the map -- 0 float atomics into 'out'; 1 float atomics into 'out' plus each
    // addition's rounding error (two-sum) into 'comp'; 2 double atomics into 'out64'.
    // max_run_lines > 0 flushes the tile at least every that many cache lines.
    int flush;
    float *comp;
    double *out64;
    int64_t max_run_lines;
    // Flush mode 3 (hot cells): hot_slot[iycell * nxcells + ixcell] >= 0 names the cell's float64
    // accumulator hot[slot][3][64][64]; partials of other cells go into 'out' as float atomics.
    const int32_t *hot_slot;
    double *hot;
    // Batches: per-TOD descriptors (owner words carry the TOD index in bits 48-63); xp, nsamp and
    // the TOD pointer of the OpArgs are then unused.
    const gmm_tod_desc *descs;
    int ntod;
    // Grid: operator CTAs per SM and minimum cache lines per CTA (0: the defaults).
    int ctas_per_sm;
    int min_lines_per_cta;
};

// Tile flush modes of OpArgs::flush.
constexpr int kFlushF32 = 0;
constexpr int kFlushCompensated = 1;
constexpr int kFlushF64 = 2;
constexpr int kFlushHotF64 = 3;
constexpr int64_t kHotCellDoubles = 3 * 64 * 64;   // one hot cell's accumulator: [3][64][64]

// Raises a kernel's dynamic shared-memory limit, once per device: 'done' holds one bit per device
// ordinal (ordinals >= 64 set it on every call).
template<typename Kernel>
cudaError_t set_smem_limit(Kernel k, size_t nbytes, std::atomic<uint64_t> &done)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return e;
    const uint64_t bit = (dev < 64) ? (1ull << dev) : 0ull;
    if (done.load(std::memory_order_acquire) & bit)
        return cudaSuccess;
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) nbytes);
    if (e == cudaSuccess)
        done.fetch_or(bit, std::memory_order_release);
    return e;
}

// Kernel of the plain planned tod2map of single-TOD plans (gmm_set_planned_tod2map_kernel).
extern int g_tod2map_kernel;

cudaError_t launch_planned_map2tod(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   cudaStream_t stream);
// 'band' (tod2map): the plan's band words, one per owner entry, or null (batch-format plans).
cudaError_t launch_planned_tod2map(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   const uint64_t *band, cudaStream_t stream);
cudaError_t launch_fold_compensation(float *lmap, float *comp, int64_t n, cudaStream_t stream);
cudaError_t launch_plan_cell_lines(const uint64_t *mt, int64_t nmt, int nycells, int nxcells, uint32_t *lines,
                                   cudaStream_t stream);
cudaError_t launch_hot_cells(const uint32_t *lines, const int64_t *cell_offsets, int ncells, uint32_t min_lines,
                             int32_t *slot, int32_t *cells, int32_t *nhot, cudaStream_t stream);
cudaError_t launch_fold_hot(float *lmap, double *hot, const int32_t *cells, int64_t nhot, const int64_t *cell_offsets,
                            int64_t ystride, int64_t polstride, cudaStream_t stream);
// Batches of TODs.
constexpr int kBatchTodShift = 48;
cudaError_t launch_batch_owner(const gmm_tod_desc *descs, int ntod, int64_t total_lines, int ny, int nx, bool periodic,
                               uint64_t *owner_out, uint32_t *cellmap, void *const *plans_each, uint32_t *errword,
                               cudaStream_t stream);
cudaError_t launch_plans_each(const gmm_tod_desc *descs, int ntod, int64_t total_lines, int ny, int nx, bool periodic,
                              void *const *plans, uint64_t *a, uint64_t *b, uint32_t *hist, int digit_bits,
                              int npasses, int tod_bits, uint32_t *errword, cudaStream_t stream);
cudaError_t launch_batch_merge(const void *const *plans, const int64_t *nlines, int ntod, int64_t total_lines,
                               uint64_t *owner_out, uint32_t *cellmap, cudaStream_t stream);
cudaError_t launch_batch_map2tod(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                 cudaStream_t stream);
cudaError_t launch_batch_tod2map(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                 cudaStream_t stream);
cudaError_t launch_unplanned_map2tod(const OpArgs &a, cudaStream_t stream);
cudaError_t launch_unplanned_tod2map(const OpArgs &a, cudaStream_t stream);

}  // namespace gmm
