// C++ API of gpu_mm_b200, mirroring the reference's include/gpu_mm.hpp (kmsmith137/gpu_mm):
// the same struct names, members and launch_* functions, with the reference's throwing,
// synchronous semantics.  It is implemented on top of the C ABI in include/gpu_mm_b200.h.
//
// Differences a C++ caller will see:
//  * Arrays are gpu_mm::Array<T>, a small strided view (data, ndim, shape, strides, size, on-GPU
//    flag, optional owner), instead of ksgpu::Array<T>.  Constructors that allocate use cudaMalloc
//    and keep the memory alive through the owner.
//  * GPU operators are provided for T = float, like the reference's Python bindings
//    (gpu_mm_pybind11.cu:17-19); the reference's float64 planned kernels cannot be launched
//    (they need 96 KB of dynamic shared memory that is never requested).
//  * PointingPrePlan::cub_nbytes keeps its name but holds the scratch size of this library's own
//    radix sort.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../gpu_mm_b200.h"

namespace gpu_mm {

typedef unsigned int uint;
typedef unsigned long ulong;

template<typename T>
struct Array {
    T *data = nullptr;
    int ndim = 0;
    long shape[4] = {0, 0, 0, 0};
    long strides[4] = {0, 0, 0, 0};   // in elements
    long size = 0;
    bool gpu = false;
    std::shared_ptr<void> base;       // keeps the memory alive (owned allocation or Python object)

    Array() = default;
    Array(T *data, const std::vector<long> &shape, bool on_gpu, std::shared_ptr<void> base = nullptr);
    Array(T *data, const std::vector<long> &shape, const std::vector<long> &strides, bool on_gpu,
          std::shared_ptr<void> base = nullptr);

    static Array<T> alloc_gpu(const std::vector<long> &shape, bool zero = false);
    static Array<T> alloc_host(const std::vector<long> &shape, bool zero = false);

    bool on_gpu() const { return gpu; }
    bool on_host() const { return !gpu; }
    bool is_fully_contiguous() const;
    std::string shape_str() const;
};

struct LocalPixelization
{
    // Python-style constructor (gpu_mm.hpp:31-35): caller keeps the CPU and GPU copies equal.
    LocalPixelization(long nypix_global, long nxpix_global,
                      const Array<long> &cell_offsets_cpu,
                      const Array<long> &cell_offsets_gpu,
                      long ystride, long polstride,
                      bool periodic_xcoord = true);

    // C++-style constructor (gpu_mm.hpp:22-25): copies 'cell_offsets' to the other side.
    LocalPixelization(long nypix_global, long nxpix_global,
                      const Array<long> &cell_offsets,
                      long ystride, long polstride,
                      bool periodic_xcoord = true);

    const long nypix_global;
    const long nxpix_global;
    const bool periodic_xcoord;

    Array<long> cell_offsets_cpu;
    Array<long> cell_offsets_gpu;
    const long ystride;
    const long polstride;

    long nycells = 0;
    long nxcells = 0;
    long npix = 0;

    void copy_gpu_offsets_to_cpu();
    void copy_cpu_offsets_to_gpu();
    void _init_npix(const char *where);

    gmm_lpix device_view() const;
};

struct PointingPrePlan
{
    static constexpr int preplan_size = GMM_PREPLAN_SIZE;

    template<typename T>
    PointingPrePlan(const Array<T> &xpointing_gpu, long nypix_global, long nxpix_global,
                    bool periodic_xcoord = true, bool debug = false);

    template<typename T>
    PointingPrePlan(const Array<T> &xpointing_gpu, long nypix_global, long nxpix_global,
                    const Array<uint> &nmt_gpu, const Array<uint> &err_gpu,
                    bool periodic_xcoord = true, bool debug = false);

    long nsamp = 0;
    long nypix_global = 0;
    long nxpix_global = 0;
    bool periodic_xcoord = true;

    long plan_nbytes = 0;
    long plan_constructor_tmp_nbytes = 0;
    double overhead = 0.0;

    long ncl_per_threadblock = 0;
    long planner_nblocks = 0;
    long nmt_per_threadblock = 0;
    long pointing_nblocks = 0;

    long plan_nmt = 0;
    size_t cub_nbytes = 0;

    Array<uint> nmt_cumsum;
    gmm_preplan_info info;

    Array<uint> get_nmt_cumsum() const;
    std::string str() const;
};

struct PointingPlan
{
    const long nsamp;
    const long nypix_global;
    const long nxpix_global;
    const bool periodic_xcoord;

    const PointingPrePlan pp;

    Array<unsigned char> buf;

    ulong *plan_mt = nullptr;
    uint *err_gpu = nullptr;
    ulong *owner_mt = nullptr;   // one word per cache line, sorted by owner cell
    ulong *band_words = nullptr; // one word per owner entry: the line's shape for the tod2map band path

    template<typename T>
    PointingPlan(const PointingPrePlan &pp, const Array<T> &xpointing_gpu,
                 const Array<unsigned char> &buf, const Array<unsigned char> &tmp_buf,
                 bool debug = false);

    template<typename T>
    PointingPlan(const PointingPrePlan &pp, const Array<T> &xpointing_gpu, bool debug = false);

    Array<ulong> get_plan_mt(bool gpu) const;
    Array<ulong> get_owner_mt(bool gpu) const;
    Array<ulong> get_band_words(bool gpu) const;
    void _check_errflags(const std::string &where) const;
    std::string str() const;
};

template<typename T>
void launch_planned_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                            const LocalPixelization &local_pixelization, const PointingPlan &plan,
                            bool partial_pixelization, bool debug, bool accum);

template<typename T>
void launch_planned_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                            const LocalPixelization &local_pixelization, const PointingPlan &plan,
                            bool partial_pixelization, bool debug);

template<typename T>
void launch_response_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                             const Array<T> &response, const LocalPixelization &local_pixelization,
                             const PointingPlan &plan, bool partial_pixelization, bool debug, bool accum);

template<typename T>
void launch_response_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                             const Array<T> &response, const LocalPixelization &local_pixelization,
                             const PointingPlan &plan, bool partial_pixelization, bool debug);

template<typename T>
void launch_unplanned_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                              const LocalPixelization &local_pixelization, Array<uint> &errflags,
                              bool partial_pixelization, bool accum);

template<typename T>
void launch_unplanned_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                              const LocalPixelization &local_pixelization, Array<uint> &errflags,
                              bool partial_pixelization);

// Precision variants of planned tod2map (no counterpart in the reference; see gpu_mm_b200.h):
// float map plus a same-size float compensation array collecting the rounding error of every float
// addition into the map (fold it in with fold_compensation), or a double map.  max_run_lines > 0
// bounds how many cache lines a partial collects before it is reduced into the map.
void launch_planned_tod2map_compensated(Array<float> &local_map, Array<float> &comp, const Array<float> &tod,
                                        const Array<float> &xpointing, const LocalPixelization &local_pixelization,
                                        const PointingPlan &plan, bool partial_pixelization, long max_run_lines = 0);
void launch_planned_tod2map_f64(Array<double> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                const LocalPixelization &local_pixelization, const PointingPlan &plan,
                                bool partial_pixelization, long max_run_lines = 0);
void fold_compensation(Array<float> &local_map, Array<float> &comp);

// float64 only for high-hit cells (no counterpart in the reference; see gpu_mm_b200.h,
// gmm_hot_cells): the cells of 'local_pixelization' touched by at least 'min_lines' cache lines of
// 'plans' (summed over the plans) reduce their tod2map partials into float64 accumulators, which
// fold() rounds into a float map once; the other cells take float atomics, as plain tod2map.
struct HotCells
{
    HotCells(const LocalPixelization &local_pixelization, const std::vector<const PointingPlan *> &plans,
             long min_lines);

    const long min_lines;
    long nycells = 0;
    long nxcells = 0;
    long nhot = 0;
    Array<uint> lines;    // (nycells, nxcells) on the GPU: cache lines of the plans touching each cell
    Array<int> slot;      // (nycells, nxcells) on the GPU: accumulator slot of each cell, -1 if not hot
    Array<int> cells;     // (nycells * nxcells,) on the GPU: cells[slot] = iycell * nxcells + ixcell
    Array<double> acc;    // (nhot, 3, 64, 64) on the GPU, zero after construction and after fold()

    // local_map += acc (one rounding per value), then acc = 0.
    void fold(Array<float> &local_map, const LocalPixelization &local_pixelization);
    // Host copies of 'lines' and 'slot'.
    Array<uint> get_lines() const;
    Array<int> get_slot() const;
};

void launch_planned_tod2map_hot_f64(Array<float> &local_map, HotCells &hot, const Array<float> &tod,
                                    const Array<float> &xpointing, const LocalPixelization &local_pixelization,
                                    const PointingPlan &plan, bool partial_pixelization, long max_run_lines = 0);

// Non-blocking forms used by batched and served callers: the device error bits are OR-ed into
// '*errword' (device memory, zeroed by the call) and checked later with check_errword(); nothing
// synchronises.  'stream' 0 is the legacy default stream.
void launch_planned_map2tod_async(Array<float> &tod, const Array<float> &local_map, const Array<float> &xpointing,
                                  const LocalPixelization &local_pixelization, const PointingPlan &plan,
                                  bool partial_pixelization, bool accum, uint *errword, cudaStream_t stream);
void launch_planned_tod2map_async(Array<float> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                  const LocalPixelization &local_pixelization, const PointingPlan &plan,
                                  bool partial_pixelization, uint *errword, cudaStream_t stream);
void launch_unplanned_map2tod_async(Array<float> &tod, const Array<float> &local_map, const Array<float> &xpointing,
                                    const LocalPixelization &local_pixelization, bool partial_pixelization,
                                    bool accum, uint *errword, cudaStream_t stream);
void launch_unplanned_tod2map_async(Array<float> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                    const LocalPixelization &local_pixelization, bool partial_pixelization,
                                    uint *errword, cudaStream_t stream);
// Waits for 'stream', reads the error word and throws the reference's message if any bit outside
// 'ignore' is set.
void check_errword(const uint *errword, uint ignore, cudaStream_t stream);

// Slow, single-threaded CPU implementations kept for API parity (gpu_mm.hpp:227-247); selected
// only explicitly (plan='reference' in Python), never as a fallback.
template<typename T>
void reference_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                       const LocalPixelization &local_pixelization, bool partial_pixelization, bool accum);

template<typename T>
void reference_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                       const LocalPixelization &local_pixelization, bool partial_pixelization);

uint expand_dynamic_map(Array<uint> &global_ncells, Array<long> &cell_offsets, const Array<ulong> &plan_mt);
uint expand_dynamic_map2(Array<uint> &global_ncells, LocalPixelization &local_pixelization, const PointingPlan &plan);

template<typename T>
void local_map_to_global(const LocalPixelization &local_pixelization, Array<T> &dst, const Array<T> &src);

// Test utilities of the reference's public surface (gpu_mm.hpp:314-430).
//
// ToyPointing: a synthetic 45-degree raster over the full y range with a slow x drift
// (ToyPointing.cu:29-117); writes xpointing_cpu, then copies it into xpointing_gpu.
template<typename T>
struct ToyPointing {
    ToyPointing(long ndet, long nt, long nypix_global, long nxpix_global, double scan_speed, double total_drift,
                bool noisy = true);
    ToyPointing(long nypix_global, long nxpix_global, double scan_speed, double total_drift,
                const Array<T> &xpointing_cpu, const Array<T> &xpointing_gpu, bool noisy = true);

    long nypix_global = 0;
    long nxpix_global = 0;
    double scan_speed = 0.0;    // map pixels per sample
    double total_drift = 0.0;   // the constructor argument
    double drift_speed = 0.0;   // x-pixels per sample: total_drift / (3 * xpointing size), as in the reference
    Array<T> xpointing_cpu;
    Array<T> xpointing_gpu;

    std::string str() const;
};

// PointingPlanTester: the plan computed the simple way, for tests (PointingPlanTester.cu:69-160).
// (iypix, ixpix) per sample come from the GPU (same roundoff as the plan); per cache line the
// distinct cells of the four neighbours, sorted, as mt words; nmt_cumsum per planner block; and all
// words sorted.  All arrays are on the host.
struct PointingPlanTester {
    PointingPlanTester(const PointingPrePlan &pp, const Array<float> &xpointing_gpu);
    PointingPlanTester(const PointingPrePlan &pp, const Array<float> &xpointing_gpu, const Array<unsigned char> &tmp);

    long nsamp = 0;
    long nypix_global = 0;
    long nxpix_global = 0;
    bool periodic_xcoord = true;
    long plan_nmt = 0;
    long ncl_per_threadblock = 0;
    long planner_nblocks = 0;

    Array<int> iypix_arr;      // length nsamp
    Array<int> ixpix_arr;      // length nsamp
    Array<uint> nmt_cumsum;    // length planner_nblocks
    Array<ulong> sorted_mt;    // length plan_nmt

    std::string str() const;
    static long get_constructor_tmp_nbytes(const PointingPrePlan &pp);
    static constexpr int nsamp_per_block = 1024;
};

// TOD preprocessing on device arrays (deglitching.cu:99-210, cuts.cu:38-55, misc.cu:8-19); index
// maps are int32.  deglitch without 'cumj' computes the jump cumsum on the device.  tod_ranges mode: 0 extract (rdata <- tod), 1 insert (tod <- rdata), 2 clear.
void get_border_means(Array<float> &out, const Array<float> &signal, const Array<int> &index_map);
void deglitch(Array<float> &signal, const Array<float> &bvals, const Array<int> &index_map2);
void deglitch(Array<float> &signal, const Array<float> &bvals, const Array<float> &cumj, const Array<int> &index_map2);
void tod_ranges(int mode, Array<float> &tod, Array<float> &rdata, const Array<int> &ostart, const Array<int> &det,
                const Array<int> &istart, const Array<int> &len);
void clip(Array<float> &arr, float vmin, float vmax);

// Cell-major buffer exchange (cell_broadcast.cu, cell_reduce.cu): dst cell i = src cell index_map[i];
// dst cell index_map[i] += src cell i (dst zeroed first).  Host arrays, or device arrays (float).
template<typename T>
void cell_broadcast(Array<T> &dst, const Array<T> &src, const Array<long> &index_map);
template<typename T>
void cell_reduce(Array<T> &dst, const Array<T> &src, const Array<long> &index_map);

// Argument checks (check_arguments.cu).
void check_nsamp(long nsamp, const char *where);
void check_nypix_global(long nypix_global, const char *where);
void check_nxpix_global(long nxpix_global, const char *where);
template<typename T> void check_tod_and_init_nsamp(const Array<T> &tod, long &nsamp, const char *where, bool on_gpu);
template<typename T> void check_xpointing_and_init_nsamp(const Array<T> &xp, long &nsamp, const char *where, bool on_gpu);
template<typename T> void check_local_map(const Array<T> &map, const LocalPixelization &lpix, const char *where, bool on_gpu);
void check_buffer(const Array<unsigned char> &buf, long min_nbytes, const char *where, const char *bufname);

// Throws std::runtime_error with gmm_last_error() if rc != 0.
void throw_on_error(int rc);

}  // namespace gpu_mm
