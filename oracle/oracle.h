/*
 * CPU oracle for the gpu_mm pointing-operator hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This library is the checker that the CUDA product path is compared against.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.  The product never calls it:
 * there is no CPU fallback.
 *
 * Every function restates the reference algorithm, citing the reference file:line it follows
 * (paths are relative to the kmsmith137/gpu_mm source tree).
 *
 * Parity pinning: the operators (locate/eval/accum loops) are pinned against oracle/_ref, which
 * compiles the reference's own include/gpu_mm_internals.hpp templates (see oracle/Makefile), and
 * against the golden vectors under tests/golden/ that were generated from it.  The plan oracle
 * restates PointingPlanTester.cu (nmt_cumsum, sorted mt multiset) and PointingPlan.cu's per-warp
 * ring buffer (mflag, zflag); the reference's plan kernels themselves need the absent ksgpu
 * library, so the zflag restatement is checked against the reference's own invariants only.
 */
#ifndef GPU_MM_ORACLE_H
#define GPU_MM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error bits, same values as gpu_mm_internals.hpp:26-29. */
#define ORACLE_ERR_BAD_YPIX 0x1u
#define ORACLE_ERR_BAD_XPIX 0x2u
#define ORACLE_ERR_INCONSISTENT_NMT 0x4u
#define ORACLE_ERR_NOT_IN_PIXELIZATION 0x8u

/* Local pixelization (gpu_mm.hpp:17-58). cell_offsets is [nycells][nxcells], -1 = absent. */
typedef struct {
    int32_t nypix_global;
    int32_t nxpix_global;
    int32_t periodic_xcoord;
    int32_t nycells;
    int32_t nxcells;
    int32_t pad_;
    int64_t ystride;
    int64_t polstride;
    const int64_t *cell_offsets;
} oracle_lpix;

/* pixel_locator<T>::locate (gpu_mm_internals.hpp:124-164). Returns error bits. */
uint32_t oracle_locate_f32(float ypix, float xpix, int32_t ny, int32_t nx, int32_t periodic,
                           int32_t out_idx[4], float out_d[2]);
uint32_t oracle_locate_f64(double ypix, double xpix, int32_t ny, int32_t nx, int32_t periodic,
                           int32_t out_idx[4], double out_d[2]);

/* reference_map2tod / reference_tod2map (map2tod_reference.cu:16-54, tod2map_reference.cu:14-46).
 * Single-threaded, sample order 0..nsamp-1, exactly like the reference.  Return error bits OR'ed
 * over all samples; partial_pixelization does NOT mask bit 8 here (caller masks). */
uint32_t oracle_map2tod_f32(float *tod, const float *lmap, const float *xpointing, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial_pixelization, int32_t accum);
uint32_t oracle_map2tod_f64(double *tod, const double *lmap, const double *xpointing, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial_pixelization, int32_t accum);
uint32_t oracle_tod2map_f32(float *lmap, const float *tod, const float *xpointing, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial_pixelization);
uint32_t oracle_tod2map_f64(double *lmap, const double *tod, const double *xpointing, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial_pixelization);

/* reference_tod2map<double> on float32 TOD/xpointing widened to double, nthreads threads with
 * private double maps summed at the end (FP64 oracle of the tod2map precision variants). */
uint32_t oracle_tod2map_f64w_mt(double *lmap, const float *tod, const float *xpointing, int64_t nsamp, int64_t map_size,
                                const oracle_lpix *lpix, int32_t partial_pixelization, int32_t nthreads);

/* Response variants (map2tod_response.cu:168-186, tod2map_response.cu:108-130): per-detector
 * (t_resp, p_resp) = (response[det], response[det+ndet]) with det = s / nperdet. */
uint32_t oracle_response_map2tod_f32(float *tod, const float *lmap, const float *xpointing,
                                     const float *response, int64_t ndet, int64_t nperdet,
                                     const oracle_lpix *lp, int32_t partial_pixelization, int32_t accum);
uint32_t oracle_response_tod2map_f32(float *lmap, const float *tod, const float *xpointing,
                                     const float *response, int64_t ndet, int64_t nperdet,
                                     const oracle_lpix *lp, int32_t partial_pixelization);

/* Same loops over a sample range [s0, s1) (used by the multi-threaded CPU baseline, which
 * gives each thread a contiguous range and, for tod2map, a private map). */
uint32_t oracle_map2tod_f32_range(float *tod, const float *lmap, const float *xpointing, int64_t nsamp,
                                  int64_t s0, int64_t s1, const oracle_lpix *lp,
                                  int32_t partial_pixelization, int32_t accum);
uint32_t oracle_tod2map_f32_range(float *lmap, const float *tod, const float *xpointing, int64_t nsamp,
                                  int64_t s0, int64_t s1, const oracle_lpix *lp, int32_t partial_pixelization);

/* Multi-threaded versions (pthreads; tod2map uses per-thread private maps then a sum). */
uint32_t oracle_map2tod_f32_mt(float *tod, const float *lmap, const float *xpointing, int64_t nsamp,
                               const oracle_lpix *lp, int32_t partial_pixelization, int32_t accum,
                               int32_t nthreads);
uint32_t oracle_tod2map_f32_mt(float *lmap, const float *tod, const float *xpointing, int64_t nsamp,
                               int64_t map_size, const oracle_lpix *lp, int32_t partial_pixelization,
                               int32_t nthreads);

/* PointingPrePlan geometry + nmt_cumsum (PointingPrePlan.cu:159-250, PointingPlanTester.cu:122-157).
 * geom_out = {ncl_per_threadblock, planner_nblocks, nmt_per_threadblock, pointing_nblocks}.
 * nmt_cumsum_out has 1024 entries (padded with the total, PointingPrePlan.cu:205-211).
 * Returns nmt (total number of mt words), or -1 if nsamp is invalid. *err_out gets locate errors. */
int64_t oracle_preplan(const float *xpointing, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                       uint32_t *nmt_cumsum_out, int64_t *geom_out, uint32_t *err_out);

/* The full plan in canonical order: mt words sorted by (cell, cache line), with mflag (bit 46)
 * and zflag (bit 47) exactly as PointingPlan.cu:60-117,167-189 produce them.  owner_bits_out
 * (ceil(nmt/32) words) marks, for each cache line, the entry with the lowest cell index.
 * Returns 0, or error bits (ORACLE_ERR_INCONSISTENT_NMT if nmt differs). */
uint32_t oracle_plan(const float *xpointing, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                     int64_t nmt, uint64_t *plan_mt_out, uint32_t *owner_bits_out);

/* Per-sample cell slots (restating cell_enumerator::enumerate), slots_out[6*nsamp], -1 = empty. */
void oracle_sample_slots(const float *xpointing, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                         int32_t *slots_out);

/* Per-line distinct-cell counts (for tests): counts_out[ncl]. */
void oracle_line_counts(const float *xpointing, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                        uint8_t *counts_out);

#ifdef __cplusplus
}
#endif

#endif
