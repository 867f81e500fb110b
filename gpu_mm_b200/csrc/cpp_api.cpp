// C++ API of gpu_mm_b200 (include/gpu_mm_b200/gpu_mm.hpp), implemented over the C ABI.
//
// Mirrors the reference's src_lib/LocalPixelization.cu, PointingPrePlan.cu (host part),
// PointingPlan.cu (host part), check_arguments.cu and the launch_* wrappers: same checks, same
// exceptions, same synchronous error-flag semantics.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <type_traits>

#include <cuda_runtime.h>

#include "../../include/gpu_mm_b200/gpu_mm.hpp"

namespace gpu_mm {

void throw_on_error(int rc)
{
    if (rc != 0)
        throw std::runtime_error(gmm_last_error());
}

static void cuda_check(cudaError_t e, const char *where)
{
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(where) + ": CUDA error: " + cudaGetErrorString(e));
}

#define GMM_ASSERT(cond, where)                                                                  \
    do {                                                                                         \
        if (!(cond))                                                                             \
            throw std::runtime_error(std::string(where) + ": assertion failed: " #cond);         \
    } while (0)

// ------------------------------------------------------------------------------------------------
// Array

template<typename T>
Array<T>::Array(T *data_, const std::vector<long> &shape_, bool on_gpu, std::shared_ptr<void> base_)
    : data(data_), gpu(on_gpu), base(std::move(base_))
{
    GMM_ASSERT(shape_.size() >= 1 && shape_.size() <= 4, "Array");
    ndim = (int) shape_.size();
    size = 1;
    for (int i = ndim - 1; i >= 0; i--) {
        shape[i] = shape_[i];
        strides[i] = size;
        size *= shape_[i];
    }
}

template<typename T>
Array<T>::Array(T *data_, const std::vector<long> &shape_, const std::vector<long> &strides_, bool on_gpu,
                std::shared_ptr<void> base_)
    : data(data_), gpu(on_gpu), base(std::move(base_))
{
    GMM_ASSERT(shape_.size() >= 1 && shape_.size() <= 4 && shape_.size() == strides_.size(), "Array");
    ndim = (int) shape_.size();
    size = 1;
    for (int i = 0; i < ndim; i++) {
        shape[i] = shape_[i];
        strides[i] = strides_[i];
        size *= shape_[i];
    }
}

template<typename T>
Array<T> Array<T>::alloc_gpu(const std::vector<long> &shape, bool zero)
{
    long n = 1;
    for (long s : shape) n *= s;
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, std::max<long>(n, 1) * sizeof(T)), "Array::alloc_gpu");
    if (zero)
        cuda_check(cudaMemset(p, 0, std::max<long>(n, 1) * sizeof(T)), "Array::alloc_gpu");
    std::shared_ptr<void> owner(p, [](void *q) { cudaFree(q); });
    return Array<T>((T *) p, shape, true, owner);
}

template<typename T>
Array<T> Array<T>::alloc_host(const std::vector<long> &shape, bool zero)
{
    long n = 1;
    for (long s : shape) n *= s;
    T *p = new T[std::max<long>(n, 1)];
    if (zero)
        std::memset((void *) p, 0, std::max<long>(n, 1) * sizeof(T));
    std::shared_ptr<void> owner((void *) p, [](void *q) { delete[] (T *) q; });
    return Array<T>(p, shape, false, owner);
}

template<typename T>
bool Array<T>::is_fully_contiguous() const
{
    long expected = 1;
    for (int i = ndim - 1; i >= 0; i--) {
        if (shape[i] != 1 && strides[i] != expected)
            return false;
        expected *= shape[i];
    }
    return true;
}

template<typename T>
std::string Array<T>::shape_str() const
{
    std::ostringstream ss;
    ss << "(";
    for (int i = 0; i < ndim; i++)
        ss << (i ? "," : "") << shape[i];
    ss << ")";
    return ss.str();
}

template struct Array<float>;
template struct Array<double>;
template struct Array<long>;
template struct Array<uint>;
template struct Array<ulong>;
template struct Array<unsigned char>;
template struct Array<int>;

// ------------------------------------------------------------------------------------------------
// Argument checks (check_arguments.cu:20-228)

void check_nsamp(long nsamp, const char *where)
{
    if ((nsamp <= 0) || (nsamp > (1L << 31)) || (nsamp % 32) != 0) {
        std::ostringstream ss;
        ss << where << ": nsamp=" << nsamp << " must be positive, <= 2^31, and a multiple of 32";
        throw std::runtime_error(ss.str());
    }
}

void check_nypix_global(long n, const char *where)
{
    if ((n <= 0) || (n > 64 * 1024))
        throw std::runtime_error(std::string(where) + ": nypix_global out of range [1, 65536]");
}

void check_nxpix_global(long n, const char *where)
{
    if ((n <= 0) || (n > 64 * 1024))
        throw std::runtime_error(std::string(where) + ": nxpix_global out of range [1, 65536]");
}

static void check_location(bool gpu, const char *where, const char *name, bool on_gpu)
{
    if (gpu == on_gpu)
        return;
    std::ostringstream ss;
    ss << where << ": expected " << name << " to be in " << (on_gpu ? "GPU" : "CPU") << " memory";
    throw std::runtime_error(ss.str());
}

template<typename T>
void check_tod_and_init_nsamp(const Array<T> &tod, long &nsamp, const char *where, bool on_gpu)
{
    GMM_ASSERT((tod.ndim == 1) || (tod.ndim == 2), where);
    GMM_ASSERT(tod.is_fully_contiguous(), where);
    nsamp = (tod.ndim == 1) ? tod.shape[0] : (tod.shape[0] * tod.shape[1]);
    check_nsamp(nsamp, where);
    check_location(tod.gpu, where, "tod", on_gpu);
}

template<typename T>
void check_xpointing_and_init_nsamp(const Array<T> &xp, long &nsamp, const char *where, bool on_gpu)
{
    GMM_ASSERT((xp.ndim == 2) || (xp.ndim == 3), where);
    GMM_ASSERT(xp.shape[0] == 3, where);
    GMM_ASSERT(xp.is_fully_contiguous(), where);
    nsamp = (xp.ndim == 2) ? xp.shape[1] : (xp.shape[1] * xp.shape[2]);
    check_nsamp(nsamp, where);
    check_location(xp.gpu, where, "xpointing", on_gpu);
}

template<typename T>
static void check_tod(const Array<T> &tod, long nsamp_expected, const char *where, bool on_gpu)
{
    long n;
    check_tod_and_init_nsamp(tod, n, where, on_gpu);
    if (n != nsamp_expected) {
        std::ostringstream ss;
        ss << where << ": tod has nsamp=" << n << ", expected " << nsamp_expected;
        throw std::runtime_error(ss.str());
    }
}

template<typename T>
static void check_xpointing(const Array<T> &xp, long nsamp_expected, const char *where, bool on_gpu)
{
    long n;
    check_xpointing_and_init_nsamp(xp, n, where, on_gpu);
    if (n != nsamp_expected) {
        std::ostringstream ss;
        ss << where << ": xpointing has nsamp=" << n << ", expected " << nsamp_expected;
        throw std::runtime_error(ss.str());
    }
}

template<typename T>
void check_local_map(const Array<T> &map, const LocalPixelization &lpix, const char *where, bool on_gpu)
{
    GMM_ASSERT(map.is_fully_contiguous(), where);
    if (map.size != 3 * lpix.npix) {
        std::ostringstream ss;
        ss << where << ": local map has size " << map.size << ", expected 3*npix = " << 3 * lpix.npix;
        throw std::runtime_error(ss.str());
    }
    check_location(map.gpu, where, "map", on_gpu);
}

void check_buffer(const Array<unsigned char> &buf, long min_nbytes, const char *where, const char *bufname)
{
    if ((buf.ndim != 1) || (buf.size < min_nbytes)) {
        std::ostringstream ss;
        ss << where << ": expected '" << bufname << "' to be 1-d array of length >= " << min_nbytes
           << ", actual shape=" << buf.shape_str();
        throw std::runtime_error(ss.str());
    }
    if (!buf.on_gpu())
        throw std::runtime_error(std::string(where) + ": array '" + bufname + "' must be on GPU");
    if (!buf.is_fully_contiguous())
        throw std::runtime_error(std::string(where) + ": array '" + bufname + "' must be contiguous");
}

static void check_cell_offsets(const Array<long> &c, long &nyc, long &nxc, const char *where, bool on_gpu)
{
    GMM_ASSERT(c.ndim == 2, where);
    GMM_ASSERT(c.is_fully_contiguous(), where);
    nyc = c.shape[0];
    nxc = c.shape[1];
    if ((nyc <= 0) || (nxc <= 0) || (nyc > 1024) || (nxc > 1024))
        throw std::runtime_error(std::string(where) + ": cell_offsets shape must be in [1,1024] x [1,1024]");
    check_location(c.gpu, where, "cell_offsets", on_gpu);
}

// ------------------------------------------------------------------------------------------------
// LocalPixelization (LocalPixelization.cu:33-101)

static Array<long> copy_offsets(const Array<long> &src, bool to_gpu)
{
    Array<long> dst = to_gpu ? Array<long>::alloc_gpu({src.shape[0], src.shape[1]})
                             : Array<long>::alloc_host({src.shape[0], src.shape[1]});
    cuda_check(cudaMemcpy(dst.data, src.data, src.size * sizeof(long), cudaMemcpyDefault), "LocalPixelization");
    return dst;
}

LocalPixelization::LocalPixelization(long ny, long nx, const Array<long> &cell_offsets, long ys, long ps, bool periodic)
    : LocalPixelization(ny, nx, cell_offsets.on_gpu() ? copy_offsets(cell_offsets, false) : cell_offsets,
                        cell_offsets.on_gpu() ? cell_offsets : copy_offsets(cell_offsets, true), ys, ps, periodic)
{ }

LocalPixelization::LocalPixelization(long ny, long nx, const Array<long> &cpu, const Array<long> &gpu_, long ys, long ps,
                                     bool periodic)
    : nypix_global(ny), nxpix_global(nx), periodic_xcoord(periodic), cell_offsets_cpu(cpu), cell_offsets_gpu(gpu_),
      ystride(ys), polstride(ps)
{
    const char *where = "LocalPixelization constructor";
    check_nypix_global(ny, where);
    check_nxpix_global(nx, where);
    check_cell_offsets(cell_offsets_cpu, nycells, nxcells, where, false);
    long nyg, nxg;
    check_cell_offsets(cell_offsets_gpu, nyg, nxg, where, true);
    if ((nyg != nycells) || (nxg != nxcells))
        throw std::runtime_error(std::string(where) + ": cell_offsets_cpu and cell_offsets_gpu shapes differ");
    GMM_ASSERT(ystride > 0, where);
    GMM_ASSERT((ystride % 64) == 0, where);
    GMM_ASSERT(polstride > 0, where);
    GMM_ASSERT((polstride % 64) == 0, where);
    const bool case1 = (ystride % (3 * polstride)) == 0;
    const bool case2 = (polstride % (64 * ystride)) == 0;
    if (!case1 && !case2)
        throw std::runtime_error("LocalPixelization constructor: expected either ystride to be a multiple of (3*polstride), or polstride to be a multiple of (64*ystride)");
    _init_npix(where);
}

void LocalPixelization::_init_npix(const char *where)
{
    // LocalPixelization.cu:74-101: cells must tile a contiguous memory region.
    long max_offset = 0;
    npix = 0;
    for (long iy = 0; iy < nycells; iy++) {
        for (long ix = 0; ix < nxcells; ix++) {
            const long off = cell_offsets_cpu.data[iy * nxcells + ix];
            if (off < 0)
                continue;
            if (off % 64)
                throw std::runtime_error(std::string(where) + ": cell offsets must be multiples of 64");
            max_offset = std::max(max_offset, off);
            npix += 64 * 64;
        }
    }
    max_offset += 2 * polstride + 63 * ystride + 63;
    if ((npix > 0) && (max_offset != (3 * npix - 1)))
        throw std::runtime_error(std::string(where) + ": something is wrong with the cell_offsets -- the cells do not fit together contiguously");
}

void LocalPixelization::copy_gpu_offsets_to_cpu()
{
    cuda_check(cudaMemcpy(cell_offsets_cpu.data, cell_offsets_gpu.data, nycells * nxcells * sizeof(long),
                          cudaMemcpyDefault), "LocalPixelization::copy_gpu_offsets_to_cpu");
    _init_npix("LocalPixelization::copy_gpu_offsets_to_cpu()");
}

void LocalPixelization::copy_cpu_offsets_to_gpu()
{
    _init_npix("LocalPixelization::copy_cpu_offsets_to_gpu");
    cuda_check(cudaMemcpy(cell_offsets_gpu.data, cell_offsets_cpu.data, nycells * nxcells * sizeof(long),
                          cudaMemcpyDefault), "LocalPixelization::copy_cpu_offsets_to_gpu");
}

gmm_lpix LocalPixelization::device_view() const
{
    gmm_lpix v;
    v.nypix_global = (int32_t) nypix_global;
    v.nxpix_global = (int32_t) nxpix_global;
    v.periodic_xcoord = periodic_xcoord ? 1 : 0;
    v.nycells = (int32_t) nycells;
    v.nxcells = (int32_t) nxcells;
    v.reserved = 0;
    v.ystride = ystride;
    v.polstride = polstride;
    v.npix = npix;
    v.cell_offsets = (const int64_t *) cell_offsets_gpu.data;
    return v;
}

// ------------------------------------------------------------------------------------------------
// PointingPrePlan (PointingPrePlan.cu:114-280)

template<typename T>
PointingPrePlan::PointingPrePlan(const Array<T> &xp, long ny, long nx, bool periodic, bool debug)
    : PointingPrePlan(xp, ny, nx, Array<uint>::alloc_gpu({preplan_size}), Array<uint>::alloc_gpu({preplan_size}),
                      periodic, debug)
{ }

template<typename T>
PointingPrePlan::PointingPrePlan(const Array<T> &xp, long ny, long nx, const Array<uint> &nmt_gpu,
                                 const Array<uint> &err_gpu, bool periodic, bool debug)
{
    static_assert(sizeof(T) == 4, "gpu_mm_b200 plans are built from float32 xpointing");
    const char *where = "PointingPrePlan constructor";
    nypix_global = ny;
    nxpix_global = nx;
    periodic_xcoord = periodic;
    nmt_cumsum = nmt_gpu;
    check_xpointing_and_init_nsamp(xp, nsamp, where, true);
    check_nypix_global(ny, where);
    check_nxpix_global(nx, where);
    GMM_ASSERT(nmt_gpu.is_fully_contiguous() && nmt_gpu.size == preplan_size && nmt_gpu.on_gpu(), where);
    GMM_ASSERT(err_gpu.is_fully_contiguous() && err_gpu.size == preplan_size && err_gpu.on_gpu(), where);

    throw_on_error(gmm_preplan((const float *) xp.data, nsamp, (int32_t) ny, (int32_t) nx, periodic ? 1 : 0,
                               (uint32_t *) nmt_gpu.data, (uint32_t *) err_gpu.data, debug ? 1 : 0, 0, &info));
    plan_nbytes = info.plan_nbytes;
    plan_constructor_tmp_nbytes = info.plan_constructor_tmp_nbytes;
    overhead = info.overhead;
    ncl_per_threadblock = info.ncl_per_threadblock;
    planner_nblocks = info.planner_nblocks;
    nmt_per_threadblock = info.nmt_per_threadblock;
    pointing_nblocks = info.pointing_nblocks;
    plan_nmt = info.plan_nmt;
    cub_nbytes = (size_t) info.sort_nbytes;
}

Array<uint> PointingPrePlan::get_nmt_cumsum() const
{
    Array<uint> ret = Array<uint>::alloc_host({planner_nblocks}, true);
    cuda_check(cudaMemcpy(ret.data, nmt_cumsum.data, planner_nblocks * sizeof(uint), cudaMemcpyDefault),
               "PointingPrePlan::get_nmt_cumsum");
    return ret;
}

static std::string nbytes_str(long n)
{
    std::ostringstream ss;
    if (n >= (1L << 30)) ss << (n / double(1L << 30)) << " GB";
    else if (n >= (1L << 20)) ss << (n / double(1L << 20)) << " MB";
    else if (n >= 1024) ss << (n / 1024.0) << " KB";
    else ss << n << " bytes";
    return ss.str();
}

std::string PointingPrePlan::str() const
{
    std::ostringstream ss;
    ss << "PointingPrePlan(nsamp=" << nsamp << ", nypix_global=" << nypix_global << ", nxpix_global=" << nxpix_global
       << ", plan_nbytes=" << plan_nbytes << " (" << nbytes_str(plan_nbytes) << ")"
       << ", tmp_nbytes=" << plan_constructor_tmp_nbytes << " (" << nbytes_str(plan_constructor_tmp_nbytes) << ")"
       << ", overhead=" << overhead << ", ncl_per_threadblock=" << ncl_per_threadblock
       << ", planner_blocks=" << planner_nblocks << ", nmt_per_threadblock=" << nmt_per_threadblock
       << ", pointing_nblocks=" << pointing_nblocks << ")";
    return ss.str();
}

// ------------------------------------------------------------------------------------------------
// PointingPlan (PointingPlan.cu:237-362)

template<typename T>
PointingPlan::PointingPlan(const PointingPrePlan &preplan, const Array<T> &xp, const Array<unsigned char> &buf_,
                           const Array<unsigned char> &tmp_buf, bool debug)
    : nsamp(preplan.nsamp), nypix_global(preplan.nypix_global), nxpix_global(preplan.nxpix_global),
      periodic_xcoord(preplan.periodic_xcoord), pp(preplan), buf(buf_)
{
    static_assert(sizeof(T) == 4, "gpu_mm_b200 plans are built from float32 xpointing");
    const char *where = "PointingPlan constructor";
    check_buffer(buf, preplan.plan_nbytes, where, "buf");
    check_buffer(tmp_buf, preplan.plan_constructor_tmp_nbytes, where, "tmp_buf");
    check_xpointing(xp, preplan.nsamp, where, true);
    gmm_plan_layout lay;
    throw_on_error(gmm_plan_layout_get(&pp.info, &lay));
    plan_mt = (ulong *) (buf.data + lay.mt_offset);
    err_gpu = (uint *) (buf.data + lay.err_offset);
    owner_mt = (ulong *) (buf.data + lay.owner_offset);
    band_words = (ulong *) (buf.data + lay.band_offset);
    throw_on_error(gmm_plan_build(&pp.info, (const uint32_t *) pp.nmt_cumsum.data, (const float *) xp.data,
                                  buf.data, buf.size, tmp_buf.data, tmp_buf.size, debug ? 1 : 0, 0));
}

template<typename T>
PointingPlan::PointingPlan(const PointingPrePlan &preplan, const Array<T> &xp, bool debug)
    : PointingPlan(preplan, xp, Array<unsigned char>::alloc_gpu({preplan.plan_nbytes}),
                   Array<unsigned char>::alloc_gpu({preplan.plan_constructor_tmp_nbytes}), debug)
{ }

Array<ulong> PointingPlan::get_plan_mt(bool gpu) const
{
    Array<ulong> ret = gpu ? Array<ulong>::alloc_gpu({pp.plan_nmt}) : Array<ulong>::alloc_host({pp.plan_nmt});
    cuda_check(cudaMemcpy(ret.data, plan_mt, pp.plan_nmt * sizeof(ulong), cudaMemcpyDefault),
               "PointingPlan::get_plan_mt");
    return ret;
}

Array<ulong> PointingPlan::get_owner_mt(bool gpu) const
{
    const long n = nsamp / 32;
    Array<ulong> ret = gpu ? Array<ulong>::alloc_gpu({n}) : Array<ulong>::alloc_host({n});
    cuda_check(cudaMemcpy(ret.data, owner_mt, n * sizeof(ulong), cudaMemcpyDefault), "PointingPlan::get_owner_mt");
    return ret;
}

Array<ulong> PointingPlan::get_band_words(bool gpu) const
{
    const long n = nsamp / 32;
    Array<ulong> ret = gpu ? Array<ulong>::alloc_gpu({n}) : Array<ulong>::alloc_host({n});
    cuda_check(cudaMemcpy(ret.data, band_words, n * sizeof(ulong), cudaMemcpyDefault), "PointingPlan::get_band_words");
    return ret;
}

void PointingPlan::_check_errflags(const std::string &where) const
{
    const long n = std::max(pp.planner_nblocks, pp.pointing_nblocks);
    std::vector<uint> h(n);
    cuda_check(cudaMemcpy(h.data(), err_gpu, n * sizeof(uint), cudaMemcpyDefault), where.c_str());
    uint err = 0;
    for (uint e : h) err |= e;
    if (err) {
        std::ostringstream ss;
        ss << where << ": plan error flags 0x" << std::hex << err;
        throw std::runtime_error(ss.str());
    }
}

std::string PointingPlan::str() const
{
    std::ostringstream ss;
    ss << "PointingPlan(nsamp=" << nsamp << ", nypix_global=" << nypix_global << ", nxpix_global=" << nxpix_global
       << ", plan_nbytes=" << pp.plan_nbytes << " (" << nbytes_str(pp.plan_nbytes) << ")"
       << ", tmp_nbytes=" << pp.plan_constructor_tmp_nbytes << " (" << nbytes_str(pp.plan_constructor_tmp_nbytes) << ")"
       << ", overhead=" << pp.overhead << ", nmt_per_threadblock=" << pp.nmt_per_threadblock
       << ", pointing_nblocks=" << pp.pointing_nblocks << ")";
    return ss.str();
}

// ------------------------------------------------------------------------------------------------
// Operators (map2tod.cu:194-272, tod2map.cu:157-226, map2tod_response.cu, tod2map_response.cu,
// map2tod_unplanned.cu:74-127, tod2map_unplanned.cu:68-121)

template<typename T>
static void check_op(const LocalPixelization &lpix, const PointingPlan &plan, const char *where)
{
    if ((lpix.nypix_global != plan.nypix_global) || (lpix.nxpix_global != plan.nxpix_global) ||
        (lpix.periodic_xcoord != plan.periodic_xcoord))
        throw std::runtime_error(std::string(where) + ": LocalPixelization and PointingPlan disagree on "
                                 "(nypix_global, nxpix_global, periodic_xcoord)");
}

template<typename T>
void launch_planned_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                            const LocalPixelization &lpix, const PointingPlan &plan, bool partial, bool debug, bool accum)
{
    (void) debug;
    if constexpr (!std::is_same_v<T, float>)
        throw std::runtime_error(std::string("launch_map2tod") + ": planned operators are float32 only (the reference instantiates "
                                 "the double kernels but cannot launch them: they need 96 KB of shared memory without "
                                 "the opt-in); use the unplanned operators for double");
    check_tod(tod, plan.nsamp, "launch_map2tod", true);
    check_local_map(local_map, lpix, "launch_map2tod", true);
    check_xpointing(xpointing, plan.nsamp, "launch_map2tod", true);
    check_op<T>(lpix, plan, "launch_map2tod");
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_map2tod((float *) tod.data, (const float *) local_map.data, (const float *) xpointing.data,
                                       &v, &plan.pp.info, plan.buf.data, partial, accum, nullptr, 0));
}

template<typename T>
void launch_planned_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                            const LocalPixelization &lpix, const PointingPlan &plan, bool partial, bool debug)
{
    (void) debug;
    if constexpr (!std::is_same_v<T, float>)
        throw std::runtime_error(std::string("launch_tod2map") + ": planned operators are float32 only (the reference instantiates "
                                 "the double kernels but cannot launch them: they need 96 KB of shared memory without "
                                 "the opt-in); use the unplanned operators for double");
    check_tod(tod, plan.nsamp, "launch_tod2map", true);
    check_local_map(local_map, lpix, "launch_tod2map", true);
    check_xpointing(xpointing, plan.nsamp, "launch_tod2map", true);
    check_op<T>(lpix, plan, "launch_tod2map");
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_tod2map((float *) local_map.data, (const float *) tod.data, (const float *) xpointing.data,
                                       &v, &plan.pp.info, plan.buf.data, partial, nullptr, 0));
}

void launch_planned_tod2map_compensated(Array<float> &local_map, Array<float> &comp, const Array<float> &tod,
                                        const Array<float> &xpointing, const LocalPixelization &lpix,
                                        const PointingPlan &plan, bool partial, long max_run_lines)
{
    const char *where = "launch_tod2map_compensated";
    check_tod(tod, plan.nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_local_map(comp, lpix, where, true);
    check_xpointing(xpointing, plan.nsamp, where, true);
    check_op<float>(lpix, plan, where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_tod2map_compensated(local_map.data, comp.data, tod.data, xpointing.data, &v,
                                                   &plan.pp.info, plan.buf.data, partial, max_run_lines, nullptr, 0));
}

void launch_planned_tod2map_f64(Array<double> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                const LocalPixelization &lpix, const PointingPlan &plan, bool partial,
                                long max_run_lines)
{
    const char *where = "launch_tod2map_f64";
    check_tod(tod, plan.nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, plan.nsamp, where, true);
    check_op<float>(lpix, plan, where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_tod2map_f64(local_map.data, tod.data, xpointing.data, &v, &plan.pp.info,
                                           plan.buf.data, partial, max_run_lines, nullptr, 0));
}

void fold_compensation(Array<float> &local_map, Array<float> &comp)
{
    GMM_ASSERT(local_map.is_fully_contiguous() && comp.is_fully_contiguous(), "fold_compensation");
    GMM_ASSERT(local_map.size == comp.size, "fold_compensation");
    check_location(local_map.gpu, "fold_compensation", "map", true);
    check_location(comp.gpu, "fold_compensation", "comp", true);
    throw_on_error(gmm_fold_compensation(local_map.data, comp.data, local_map.size, 0));
    cuda_check(cudaStreamSynchronize(0), "fold_compensation");
}

HotCells::HotCells(const LocalPixelization &lpix, const std::vector<const PointingPlan *> &plans, long min_lines_)
    : min_lines(min_lines_), nycells(lpix.nycells), nxcells(lpix.nxcells)
{
    const char *where = "HotCells";
    GMM_ASSERT((min_lines >= 0) && (min_lines <= 0xffffffffl), where);
    const long ncells = nycells * nxcells;
    lines = Array<uint>::alloc_gpu({nycells, nxcells}, true);
    slot = Array<int>::alloc_gpu({nycells, nxcells});
    cells = Array<int>::alloc_gpu({ncells});
    gmm_lpix v = lpix.device_view();
    for (const PointingPlan *plan : plans) {
        GMM_ASSERT(plan != nullptr, where);
        throw_on_error(gmm_plan_cell_lines(&plan->pp.info, plan->buf.data, &v, lines.data, 0));
    }
    Array<int> n = Array<int>::alloc_gpu({1}, true);
    throw_on_error(gmm_hot_cells(lines.data, &v, (uint32_t) min_lines, slot.data, cells.data, n.data, 0));
    int h = 0;
    cuda_check(cudaMemcpy(&h, n.data, sizeof(int), cudaMemcpyDeviceToHost), where);
    nhot = h;
    acc = Array<double>::alloc_gpu({nhot, 3, 64, 64}, true);
}

void HotCells::fold(Array<float> &local_map, const LocalPixelization &lpix)
{
    const char *where = "HotCells::fold";
    check_local_map(local_map, lpix, where, true);
    GMM_ASSERT((lpix.nycells == nycells) && (lpix.nxcells == nxcells), where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_fold_hot_f64(local_map.data, acc.data, cells.data, nhot, &v, 0));
    cuda_check(cudaStreamSynchronize(0), where);
}

Array<uint> HotCells::get_lines() const
{
    Array<uint> h = Array<uint>::alloc_host({nycells, nxcells});
    cuda_check(cudaMemcpy(h.data, lines.data, h.size * sizeof(uint), cudaMemcpyDeviceToHost), "HotCells::get_lines");
    return h;
}

Array<int> HotCells::get_slot() const
{
    Array<int> h = Array<int>::alloc_host({nycells, nxcells});
    cuda_check(cudaMemcpy(h.data, slot.data, h.size * sizeof(int), cudaMemcpyDeviceToHost), "HotCells::get_slot");
    return h;
}

void launch_planned_tod2map_hot_f64(Array<float> &local_map, HotCells &hot, const Array<float> &tod,
                                    const Array<float> &xpointing, const LocalPixelization &lpix,
                                    const PointingPlan &plan, bool partial, long max_run_lines)
{
    const char *where = "launch_tod2map_hot_f64";
    check_tod(tod, plan.nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, plan.nsamp, where, true);
    check_op<float>(lpix, plan, where);
    GMM_ASSERT((lpix.nycells == hot.nycells) && (lpix.nxcells == hot.nxcells), where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_tod2map_hot_f64(local_map.data, hot.acc.data, hot.slot.data, tod.data, xpointing.data,
                                               &v, &plan.pp.info, plan.buf.data, partial, max_run_lines, nullptr, 0));
}

template<typename T>
static long check_response(const Array<T> &response, long nsamp, const char *where)
{
    // check_arguments.cu:171-180: response has shape (2, ndet) and ndet divides nsamp.
    GMM_ASSERT(response.ndim == 2, where);
    GMM_ASSERT(response.shape[0] == 2, where);
    GMM_ASSERT(response.is_fully_contiguous(), where);
    const long ndet = response.shape[1];
    GMM_ASSERT(ndet > 0 && (nsamp % ndet) == 0, where);
    check_location(response.gpu, where, "response", true);
    return ndet;
}

template<typename T>
void launch_response_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing, const Array<T> &response,
                             const LocalPixelization &lpix, const PointingPlan &plan, bool partial, bool debug, bool accum)
{
    (void) debug;
    if constexpr (!std::is_same_v<T, float>)
        throw std::runtime_error(std::string("launch_response_map2tod") + ": planned operators are float32 only (the reference instantiates "
                                 "the double kernels but cannot launch them: they need 96 KB of shared memory without "
                                 "the opt-in); use the unplanned operators for double");
    const char *where = "launch_response_map2tod";
    check_tod(tod, plan.nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, plan.nsamp, where, true);
    const long ndet = check_response(response, plan.nsamp, where);
    check_op<T>(lpix, plan, where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_response_map2tod((float *) tod.data, (const float *) local_map.data, (const float *) xpointing.data,
                                        (const float *) response.data, ndet, &v, &plan.pp.info, plan.buf.data, partial,
                                        accum, nullptr, 0));
}

template<typename T>
void launch_response_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing, const Array<T> &response,
                             const LocalPixelization &lpix, const PointingPlan &plan, bool partial, bool debug)
{
    (void) debug;
    if constexpr (!std::is_same_v<T, float>)
        throw std::runtime_error(std::string("launch_response_tod2map") + ": planned operators are float32 only (the reference instantiates "
                                 "the double kernels but cannot launch them: they need 96 KB of shared memory without "
                                 "the opt-in); use the unplanned operators for double");
    const char *where = "launch_response_tod2map";
    check_tod(tod, plan.nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, plan.nsamp, where, true);
    const long ndet = check_response(response, plan.nsamp, where);
    check_op<T>(lpix, plan, where);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_response_tod2map((float *) local_map.data, (const float *) tod.data, (const float *) xpointing.data,
                                        (const float *) response.data, ndet, &v, &plan.pp.info, plan.buf.data, partial,
                                        nullptr, 0));
}

static void check_errflags_arr(const Array<uint> &errflags, const char *where)
{
    GMM_ASSERT(errflags.ndim == 1, where);
    GMM_ASSERT(errflags.is_fully_contiguous(), where);
    GMM_ASSERT(errflags.on_gpu(), where);
    GMM_ASSERT(errflags.size >= 1, where);
}

template<typename T>
void launch_unplanned_map2tod(Array<T> &tod, const Array<T> &local_map, const Array<T> &xpointing,
                              const LocalPixelization &lpix, Array<uint> &errflags, bool partial, bool accum)
{
    const char *where = "unplanned_map2tod";
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, nsamp, where, true);
    check_errflags_arr(errflags, where);
    gmm_lpix v = lpix.device_view();
    if constexpr (std::is_same_v<T, double>)
        throw_on_error(gmm_unplanned_map2tod_f64(tod.data, local_map.data, xpointing.data, nsamp, &v,
                                                 (uint32_t *) errflags.data, errflags.size, partial, accum, 1, 0));
    else
        throw_on_error(gmm_unplanned_map2tod(tod.data, local_map.data, xpointing.data, nsamp, &v,
                                             (uint32_t *) errflags.data, errflags.size, partial, accum, 1, 0));
}

template<typename T>
void launch_unplanned_tod2map(Array<T> &local_map, const Array<T> &tod, const Array<T> &xpointing,
                              const LocalPixelization &lpix, Array<uint> &errflags, bool partial)
{
    const char *where = "unplanned_tod2map";
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, where, true);
    check_local_map(local_map, lpix, where, true);
    check_xpointing(xpointing, nsamp, where, true);
    check_errflags_arr(errflags, where);
    gmm_lpix v = lpix.device_view();
    if constexpr (std::is_same_v<T, double>)
        throw_on_error(gmm_unplanned_tod2map_f64(local_map.data, tod.data, xpointing.data, nsamp, &v,
                                                 (uint32_t *) errflags.data, errflags.size, partial, 1, 0));
    else
        throw_on_error(gmm_unplanned_tod2map(local_map.data, tod.data, xpointing.data, nsamp, &v,
                                             (uint32_t *) errflags.data, errflags.size, partial, 1, 0));
}

void launch_planned_map2tod_async(Array<float> &tod, const Array<float> &local_map, const Array<float> &xpointing,
                                  const LocalPixelization &lpix, const PointingPlan &plan, bool partial, bool accum,
                                  uint *errword, cudaStream_t stream)
{
    check_tod(tod, plan.nsamp, "launch_map2tod", true);
    check_local_map(local_map, lpix, "launch_map2tod", true);
    check_xpointing(xpointing, plan.nsamp, "launch_map2tod", true);
    check_op<float>(lpix, plan, "launch_map2tod");
    GMM_ASSERT(errword != nullptr, "launch_map2tod");
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_map2tod(tod.data, local_map.data, xpointing.data, &v, &plan.pp.info, plan.buf.data,
                                       partial, accum, (uint32_t *) errword, stream));
}

void launch_planned_tod2map_async(Array<float> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                  const LocalPixelization &lpix, const PointingPlan &plan, bool partial, uint *errword,
                                  cudaStream_t stream)
{
    check_tod(tod, plan.nsamp, "launch_tod2map", true);
    check_local_map(local_map, lpix, "launch_tod2map", true);
    check_xpointing(xpointing, plan.nsamp, "launch_tod2map", true);
    check_op<float>(lpix, plan, "launch_tod2map");
    GMM_ASSERT(errword != nullptr, "launch_tod2map");
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_planned_tod2map(local_map.data, tod.data, xpointing.data, &v, &plan.pp.info, plan.buf.data,
                                       partial, (uint32_t *) errword, stream));
}

void launch_unplanned_map2tod_async(Array<float> &tod, const Array<float> &local_map, const Array<float> &xpointing,
                                    const LocalPixelization &lpix, bool partial, bool accum, uint *errword,
                                    cudaStream_t stream)
{
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, "unplanned_map2tod", true);
    check_local_map(local_map, lpix, "unplanned_map2tod", true);
    check_xpointing(xpointing, nsamp, "unplanned_map2tod", true);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_unplanned_map2tod(tod.data, local_map.data, xpointing.data, nsamp, &v, (uint32_t *) errword, 1,
                                         partial, accum, 0, stream));
}

void launch_unplanned_tod2map_async(Array<float> &local_map, const Array<float> &tod, const Array<float> &xpointing,
                                    const LocalPixelization &lpix, bool partial, uint *errword, cudaStream_t stream)
{
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, "unplanned_tod2map", true);
    check_local_map(local_map, lpix, "unplanned_tod2map", true);
    check_xpointing(xpointing, nsamp, "unplanned_tod2map", true);
    gmm_lpix v = lpix.device_view();
    throw_on_error(gmm_unplanned_tod2map(local_map.data, tod.data, xpointing.data, nsamp, &v, (uint32_t *) errword, 1,
                                         partial, 0, stream));
}

void check_errword(const uint *errword, uint ignore, cudaStream_t stream)
{
    throw_on_error(gmm_errword_read((const uint32_t *) errword, ignore, stream));
}

// ------------------------------------------------------------------------------------------------
// Explicit-request CPU operators (map2tod_reference.cu:16-54, tod2map_reference.cu:14-46).

template<typename T>
static void cpu_locate(T ypix, T xpix, long ny, long nx, bool periodic, int &iy0, int &iy1, int &ix0, int &ix1,
                       T &dy, T &dx, uint &err)
{
    iy0 = (int) ypix;
    iy0 = std::max(iy0, 0);
    iy0 = std::min(iy0, (int) ny - 2);
    iy1 = iy0 + 1;
    dy = ypix - iy0;
    if (!((ypix >= 0) && (ypix <= ny - 1))) err |= GMM_ERR_BAD_YPIX;
    if (periodic) {
        if (!((xpix >= -nx) && (xpix <= 2 * nx))) err |= GMM_ERR_BAD_XPIX;
        xpix = (xpix >= 0) ? xpix : (xpix + nx);
        xpix = (xpix <= nx) ? xpix : (xpix - nx);
        ix0 = std::max((int) xpix, 0);
        dx = xpix - ix0;
        ix0 = (ix0 < nx) ? ix0 : 0;
        ix1 = (ix0 + 1 < nx) ? (ix0 + 1) : 0;
    } else {
        if (!((xpix >= 0) && (xpix <= nx - 2))) err |= GMM_ERR_BAD_XPIX;
        ix0 = std::min(std::max((int) xpix, 0), (int) nx - 2);
        ix1 = ix0 + 1;
        dx = xpix - ix0;
    }
}

static inline void cpu_sincos(float x, float *s, float *c) { ::sincosf(x, s, c); }
static inline void cpu_sincos(double x, double *s, double *c) { ::sincos(x, s, c); }

static long cpu_offset(const LocalPixelization &lp, int iy, int ix)
{
    const int iyc = iy >> 6, ixc = ix >> 6;
    if ((iy < 0) || (ix < 0) || (iyc >= lp.nycells) || (ixc >= lp.nxcells))
        return -1;
    const long off = lp.cell_offsets_cpu.data[(long) iyc * lp.nxcells + ixc];
    return (off < 0) ? -1 : (off + (ix - (ixc << 6)) + (long) (iy - (iyc << 6)) * lp.ystride);
}

template<typename T>
void reference_map2tod(Array<T> &tod, const Array<T> &lmap, const Array<T> &xp, const LocalPixelization &lp,
                       bool partial, bool accum)
{
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, "reference_map2tod", false);
    check_local_map(lmap, lp, "reference_map2tod", false);
    check_xpointing(xp, nsamp, "reference_map2tod", false);
    uint err = 0;
    for (long s = 0; s < nsamp; s++) {
        const T y = xp.data[s], x = xp.data[s + nsamp], a = xp.data[s + 2 * nsamp];
        T sn, cs;
        cpu_sincos(2 * a, &sn, &cs);
        int iy[2], ix[2];
        T dy, dx;
        cpu_locate(y, x, lp.nypix_global, lp.nxpix_global, lp.periodic_xcoord, iy[0], iy[1], ix[0], ix[1], dy, dx, err);
        const T wy[2] = {1 - dy, dy}, wx[2] = {1 - dx, dx};
        T r = 0;
        for (int a2 = 0; a2 < 2; a2++)
            for (int b2 = 0; b2 < 2; b2++) {
                const long off = cpu_offset(lp, iy[a2], ix[b2]);
                const bool valid = off >= 0;
                const T v = valid ? (lmap.data[off] + cs * lmap.data[off + lp.polstride] + sn * lmap.data[off + 2 * lp.polstride]) : T(0);
                if (!valid && !partial) err |= GMM_ERR_NOT_IN_PIXELIZATION;
                r += wy[a2] * wx[b2] * v;
            }
        tod.data[s] = accum ? (tod.data[s] + r) : r;
    }
    if (err) {
        // Same messages as check_err (check_arguments.cu:42-58).
        if (err & GMM_ERR_BAD_YPIX) throw std::runtime_error("reference_map2tod: xpointing y-value is outside range [1,nypix_global-2].");
        if (err & GMM_ERR_BAD_XPIX) throw std::runtime_error("reference_map2tod: xpointing x-value is outside range, perhaps you want the 'periodic_xcoord' flag?");
        throw std::runtime_error("reference_map2tod: xpointing (y,x) value is not in LocalPixelization (perhaps pixelization is too small, or you want the 'partial_pixelization' flag");
    }
}

template<typename T>
void reference_tod2map(Array<T> &lmap, const Array<T> &tod, const Array<T> &xp, const LocalPixelization &lp, bool partial)
{
    long nsamp;
    check_tod_and_init_nsamp(tod, nsamp, "reference_tod2map", false);
    check_local_map(lmap, lp, "reference_tod2map", false);
    check_xpointing(xp, nsamp, "reference_tod2map", false);
    uint err = 0;
    for (long s = 0; s < nsamp; s++) {
        const T y = xp.data[s], x = xp.data[s + nsamp], a = xp.data[s + 2 * nsamp];
        const T t = tod.data[s];
        T sn, cs;
        cpu_sincos(2 * a, &sn, &cs);
        int iy[2], ix[2];
        T dy, dx;
        cpu_locate(y, x, lp.nypix_global, lp.nxpix_global, lp.periodic_xcoord, iy[0], iy[1], ix[0], ix[1], dy, dx, err);
        const T wy[2] = {1 - dy, dy}, wx[2] = {1 - dx, dx};
        for (int a2 = 0; a2 < 2; a2++)
            for (int b2 = 0; b2 < 2; b2++) {
                const long off = cpu_offset(lp, iy[a2], ix[b2]);
                const T w = wy[a2] * wx[b2];
                if (off >= 0) {
                    lmap.data[off] += w * t;
                    lmap.data[off + lp.polstride] += w * (t * cs);
                    lmap.data[off + 2 * lp.polstride] += w * (t * sn);
                } else if (!partial) {
                    err |= GMM_ERR_NOT_IN_PIXELIZATION;
                }
            }
    }
    if (err) {
        if (err & GMM_ERR_BAD_YPIX) throw std::runtime_error("reference_tod2map: xpointing y-value is outside range [1,nypix_global-2].");
        if (err & GMM_ERR_BAD_XPIX) throw std::runtime_error("reference_tod2map: xpointing x-value is outside range, perhaps you want the 'periodic_xcoord' flag?");
        throw std::runtime_error("reference_tod2map: xpointing (y,x) value is not in LocalPixelization (perhaps pixelization is too small, or you want the 'partial_pixelization' flag");
    }
}

// ------------------------------------------------------------------------------------------------
// Dynamic maps and output format

uint expand_dynamic_map(Array<uint> &global_ncells, Array<long> &cell_offsets, const Array<ulong> &plan_mt)
{
    const char *where = "expand_dynamic_map";
    GMM_ASSERT(global_ncells.on_gpu() && global_ncells.size == 1, where);
    long nyc, nxc;
    check_cell_offsets(cell_offsets, nyc, nxc, where, true);
    GMM_ASSERT(plan_mt.on_gpu() && plan_mt.ndim == 1 && plan_mt.is_fully_contiguous(), where);
    uint32_t n = 0;
    throw_on_error(gmm_expand_dynamic_map((uint32_t *) global_ncells.data, (int64_t *) cell_offsets.data, (int32_t) nyc,
                                          (int32_t) nxc, (const uint64_t *) plan_mt.data, plan_mt.shape[0], &n, 0));
    return n;
}

uint expand_dynamic_map2(Array<uint> &global_ncells, LocalPixelization &lpix, const PointingPlan &plan)
{
    GMM_ASSERT(lpix.nypix_global == plan.nypix_global, "expand_dynamic_map2");
    GMM_ASSERT(lpix.nxpix_global == plan.nxpix_global, "expand_dynamic_map2");
    GMM_ASSERT(lpix.periodic_xcoord == plan.periodic_xcoord, "expand_dynamic_map2");
    Array<ulong> mt(plan.plan_mt, {plan.pp.plan_nmt}, true);
    return expand_dynamic_map(global_ncells, lpix.cell_offsets_gpu, mt);
}

template<typename T>
void local_map_to_global(const LocalPixelization &lp, Array<T> &dst, const Array<T> &src)
{
    // local_map_to_global.cu:11-45.  Host arrays: the reference's loop (dst is zeroed by the caller).
    // Device arrays (float): gmm_local_map_to_global, which also zeroes the pixels of absent cells.
    const long ny = lp.nypix_global, nx = lp.nxpix_global;
    GMM_ASSERT(dst.ndim == 3 && dst.shape[0] == 3 && dst.shape[1] == ny && dst.shape[2] == nx, "local_map_to_global");
    GMM_ASSERT(dst.is_fully_contiguous(), "local_map_to_global");
    if (dst.gpu || src.gpu) {
        GMM_ASSERT(dst.gpu && src.gpu && (sizeof(T) == sizeof(float)), "local_map_to_global");
        check_local_map(src, lp, "local_map_to_global", true);
        gmm_lpix v = lp.device_view();
        throw_on_error(gmm_local_map_to_global((float *) dst.data, (const float *) src.data, &v, 0));
        cuda_check(cudaStreamSynchronize(0), "local_map_to_global");
        return;
    }
    check_local_map(src, lp, "local_map_to_global", false);
    for (long iyc = 0; iyc < lp.nycells; iyc++)
        for (long ixc = 0; ixc < lp.nxcells; ixc++) {
            const long off = lp.cell_offsets_cpu.data[iyc * lp.nxcells + ixc];
            if (off < 0)
                continue;
            const long y0 = 64 * iyc, x0 = 64 * ixc;
            const long nyy = std::min(ny, y0 + 64) - y0, nxx = std::min(nx, x0 + 64) - x0;
            for (int p = 0; p < 3; p++)
                for (long iy = 0; iy < nyy; iy++)
                    for (long ix = 0; ix < nxx; ix++)
                        dst.data[p * ny * nx + (y0 + iy) * nx + x0 + ix] = src.data[off + p * lp.polstride + iy * lp.ystride + ix];
        }
}

// cell_broadcast.cu:17-36 / cell_reduce.cu:17-41: cell-major buffers (3*64*64 values per cell).
// Host arrays: the reference's loops and checks.  Device arrays (float): gmm_cell_broadcast /
// gmm_cell_reduce, after the same checks on a host copy of index_map.
static constexpr long kCellN = 3 * 64 * 64;

template<typename T>
static void check_cell_args(const Array<T> &dst, const Array<T> &src, const Array<long> &index_map, const char *where)
{
    GMM_ASSERT(dst.ndim == 1 && dst.is_fully_contiguous(), where);
    GMM_ASSERT(src.ndim == 1 && src.is_fully_contiguous(), where);
    GMM_ASSERT(index_map.ndim == 1 && index_map.is_fully_contiguous(), where);
    GMM_ASSERT((dst.gpu == src.gpu) && (dst.gpu == index_map.gpu), where);
    GMM_ASSERT(!dst.gpu || (sizeof(T) == sizeof(float)), where);
}

static std::vector<long> host_index_map(const Array<long> &index_map)
{
    if (!index_map.gpu)
        return std::vector<long>(index_map.data, index_map.data + index_map.size);
    std::vector<long> h(index_map.size);
    if (index_map.size > 0)
        cuda_check(cudaMemcpy(h.data(), index_map.data, index_map.size * sizeof(long), cudaMemcpyDeviceToHost),
                   "cell index_map");
    return h;
}

template<typename T>
void cell_broadcast(Array<T> &dst, const Array<T> &src, const Array<long> &index_map)
{
    check_cell_args(dst, src, index_map, "cell_broadcast");
    const long ncells = index_map.size, nsrc = src.size;
    GMM_ASSERT(dst.size == ncells * kCellN, "cell_broadcast");
    const std::vector<long> im = host_index_map(index_map);
    for (long i = 0; i < ncells; i++)
        GMM_ASSERT((im[i] >= 0) && (im[i] * kCellN + kCellN <= nsrc), "cell_broadcast");
    if (dst.gpu) {
        Array<uint> err = Array<uint>::alloc_gpu({1}, true);
        throw_on_error(gmm_cell_broadcast((float *) dst.data, (const float *) src.data, nsrc, index_map.data, ncells,
                                          (uint32_t *) err.data, 0));
        check_errword(err.data, 0, 0);
        return;
    }
    for (long i = 0; i < ncells; i++)
        std::memcpy(dst.data + i * kCellN, src.data + im[i] * kCellN, kCellN * sizeof(T));
}

template<typename T>
void cell_reduce(Array<T> &dst, const Array<T> &src, const Array<long> &index_map)
{
    check_cell_args(dst, src, index_map, "cell_reduce");
    const long ncells = index_map.size, ndst = dst.size;
    GMM_ASSERT(src.size == ncells * kCellN, "cell_reduce");
    const std::vector<long> im = host_index_map(index_map);
    for (long i = 0; i < ncells; i++)
        GMM_ASSERT((im[i] >= 0) && (im[i] * kCellN + kCellN <= ndst), "cell_reduce");
    if (dst.gpu) {
        Array<uint> err = Array<uint>::alloc_gpu({1}, true);
        throw_on_error(gmm_cell_reduce((float *) dst.data, ndst, (const float *) src.data, index_map.data, ncells,
                                       (uint32_t *) err.data, 0));
        check_errword(err.data, 0, 0);
        return;
    }
    std::memset(dst.data, 0, ndst * sizeof(T));
    for (long i = 0; i < ncells; i++) {
        T *d = dst.data + im[i] * kCellN;
        const T *q = src.data + i * kCellN;
        for (long j = 0; j < kCellN; j++)
            d[j] += q[j];
    }
}

template void cell_broadcast<float>(Array<float> &, const Array<float> &, const Array<long> &);
template void cell_broadcast<double>(Array<double> &, const Array<double> &, const Array<long> &);
template void cell_reduce<float>(Array<float> &, const Array<float> &, const Array<long> &);
template void cell_reduce<double>(Array<double> &, const Array<double> &, const Array<long> &);

// ---- Test utilities: ToyPointing, PointingPlanTester -------------------------------------------

template<typename T>
static Array<T> toy_xpointing(long ndet, long nt, bool gpu)
{
    if ((nt <= 0) || ((ndet > 0) && (ndet * nt <= 0)))
        throw std::runtime_error("ToyPointing constructor: bad (ndet, nt)");
    std::vector<long> shape = (ndet <= 0) ? std::vector<long>{3, nt} : std::vector<long>{3, ndet, nt};
    return gpu ? Array<T>::alloc_gpu(shape) : Array<T>::alloc_host(shape);
}

template<typename T>
ToyPointing<T>::ToyPointing(long ndet, long nt, long ny, long nx, double speed, double drift, bool noisy)
    : ToyPointing(ny, nx, speed, drift, toy_xpointing<T>(ndet, nt, false), toy_xpointing<T>(ndet, nt, true), noisy)
{
}

// The raster of ToyPointing.cu:63-108: y bounces between 1.1*speed and ny-2-1.1*speed at 'speed'
// pixels per sample, x moves by the same step plus the drift and wraps into [0, nx]; alpha = 1.
// Accumulated in double, as there, and stored as T.
template<typename T>
ToyPointing<T>::ToyPointing(long ny, long nx, double speed, double drift, const Array<T> &xp_cpu, const Array<T> &xp_gpu,
                            bool noisy)
    : nypix_global(ny), nxpix_global(nx), scan_speed(speed), total_drift(drift),
      drift_speed(drift / (3.0 * (double) xp_cpu.size)), xpointing_cpu(xp_cpu), xpointing_gpu(xp_gpu)
{
    const char *where = "ToyPointing constructor";
    long nsamp;
    check_xpointing_and_init_nsamp(xpointing_cpu, nsamp, where, false);
    check_xpointing(xpointing_gpu, nsamp, where, true);
    GMM_ASSERT(xpointing_cpu.is_fully_contiguous() && xpointing_gpu.is_fully_contiguous(), where);
    GMM_ASSERT((ny >= 2) && (ny <= (1 << 16)) && (nx >= 2) && (nx <= (1 << 16)), where);
    GMM_ASSERT((scan_speed > 0.0) && (scan_speed <= 1.0), where);
    GMM_ASSERT((drift_speed > 0.0) && (drift_speed <= 1.0), where);
    if (noisy)
        std::printf("%s: constructor called\n", str().c_str());
    T *yp = xpointing_cpu.data, *xp = yp + nsamp, *ap = yp + 2 * nsamp;
    const double ylo = 1.1 * speed, yhi = (double) (ny - 2) - 1.1 * speed;
    double y = 1.0, x = 1.0, vel = speed;
    for (long s = 0; s < nsamp; s++) {
        yp[s] = (T) y;
        xp[s] = (T) x;
        ap[s] = (T) 1.0;
        if ((vel > 0) && (y > yhi))
            vel = -speed;
        if ((vel < 0) && (y < ylo))
            vel = speed;
        y += vel;
        x += vel + drift_speed;
        if (x < 0.0)
            x += (double) nx;
        if (x > (double) nx)
            x -= (double) nx;
    }
    cuda_check(cudaMemcpy(xpointing_gpu.data, xpointing_cpu.data, 3 * nsamp * sizeof(T), cudaMemcpyHostToDevice), where);
    if (noisy)
        std::printf("%s: constructor done\n", str().c_str());
}

template<typename T>
std::string ToyPointing<T>::str() const
{
    std::ostringstream ss;
    ss << "ToyPointing(tod_shape=(";
    for (int i = 1; i < xpointing_cpu.ndim; i++)
        ss << (i > 1 ? "," : "") << xpointing_cpu.shape[i];
    ss << "), nypix_global=" << nypix_global << ", nxpix_global=" << nxpix_global << ", scan_speed=" << scan_speed
       << ", total_drift=" << total_drift << ")";
    return ss.str();
}

template struct ToyPointing<float>;
template struct ToyPointing<double>;

long PointingPlanTester::get_constructor_tmp_nbytes(const PointingPrePlan &pp)
{
    // The reference's size (PointingPlanTester.cu:172-178): two int arrays and one error word per block.
    const long nblocks = (pp.nsamp + nsamp_per_block - 1) / nsamp_per_block;
    return (2 * pp.nsamp + nblocks) * (long) sizeof(int);
}

PointingPlanTester::PointingPlanTester(const PointingPrePlan &pp, const Array<float> &xp)
    : PointingPlanTester(pp, xp, Array<unsigned char>::alloc_gpu({get_constructor_tmp_nbytes(pp)}))
{
}

PointingPlanTester::PointingPlanTester(const PointingPrePlan &pp, const Array<float> &xp, const Array<unsigned char> &tmp)
    : nsamp(pp.nsamp), nypix_global(pp.nypix_global), nxpix_global(pp.nxpix_global), periodic_xcoord(pp.periodic_xcoord),
      plan_nmt(pp.plan_nmt), ncl_per_threadblock(pp.ncl_per_threadblock), planner_nblocks(pp.planner_nblocks)
{
    const char *where = "PointingPlanTester constructor";
    check_xpointing(xp, nsamp, where, true);
    GMM_ASSERT(tmp.on_gpu() && tmp.is_fully_contiguous() && (tmp.size >= get_constructor_tmp_nbytes(pp)), where);
    GMM_ASSERT((nsamp > (planner_nblocks - 1) * ncl_per_threadblock * 32) &&
               (nsamp <= planner_nblocks * ncl_per_threadblock * 32), where);

    int32_t *iy_gpu = (int32_t *) tmp.data;
    int32_t *ix_gpu = iy_gpu + nsamp;
    uint32_t *err_gpu = (uint32_t *) (ix_gpu + nsamp);
    throw_on_error(gmm_quantize_pointing(xp.data, nsamp, (int32_t) nypix_global, (int32_t) nxpix_global,
                                         periodic_xcoord, iy_gpu, ix_gpu, err_gpu, 0));
    throw_on_error(gmm_errword_read(err_gpu, 0, 0));
    iypix_arr = Array<int>::alloc_host({nsamp});
    ixpix_arr = Array<int>::alloc_host({nsamp});
    cuda_check(cudaMemcpy(iypix_arr.data, iy_gpu, nsamp * sizeof(int), cudaMemcpyDeviceToHost), where);
    cuda_check(cudaMemcpy(ixpix_arr.data, ix_gpu, nsamp * sizeof(int), cudaMemcpyDeviceToHost), where);

    // Per cache line: the distinct cells of the four neighbours of its samples, ascending, as mt words
    // cell | line << 20 (PointingPlanTester.cu:126-160; x+1 wraps to 0 at the last column).
    nmt_cumsum = Array<uint>::alloc_host({planner_nblocks});
    sorted_mt = Array<ulong>::alloc_host({std::max<long>(plan_nmt, 1)});
    std::vector<int> cells;
    long n = 0;
    for (long b = 0; b < planner_nblocks; b++) {
        const long l1 = std::min(nsamp, (b + 1) * ncl_per_threadblock * 32) >> 5;
        for (long l = b * ncl_per_threadblock; l < l1; l++) {
            cells.clear();
            for (long s = 32 * l; s < 32 * l + 32; s++) {
                const int iy = iypix_arr.data[s], ix = ixpix_arr.data[s];
                const int ix1 = (ix < nxpix_global - 1) ? (ix + 1) : 0;
                for (int dy = 0; dy < 2; dy++)
                    for (int c = 0; c < 2; c++) {
                        const int cell = (((iy + dy) >> 6) << 10) | ((c ? ix1 : ix) >> 6);
                        if (std::find(cells.begin(), cells.end(), cell) == cells.end())
                            cells.push_back(cell);
                    }
            }
            std::sort(cells.begin(), cells.end());
            for (int cell : cells) {
                if (n >= plan_nmt)
                    throw std::runtime_error(std::string(where) + ": more (cell, cache line) pairs than the preplan's nmt");
                sorted_mt.data[n++] = (ulong) cell | ((ulong) l << 20);
            }
        }
        nmt_cumsum.data[b] = (uint) n;
    }
    if (n != plan_nmt)
        throw std::runtime_error(std::string(where) + ": (cell, cache line) count differs from the preplan's nmt");
    std::sort(sorted_mt.data, sorted_mt.data + n);
    sorted_mt.shape[0] = sorted_mt.size = n;
}

std::string PointingPlanTester::str() const
{
    std::ostringstream ss;
    ss << "PointingPlanTester(nsamp=" << nsamp << ", nypix_global=" << nypix_global << ", nxpix_global=" << nxpix_global
       << ", plan_nmt=" << plan_nmt << ")";
    return ss.str();
}

// ---- TOD preprocessing (deglitching.cu, cuts.cu, misc.cu): device arrays; index-map entries out of
// range raise after the call.

static void check_range_word(const Array<uint> &w, const char *where)
{
    uint h = 0;
    cuda_check(cudaMemcpy(&h, w.data, sizeof(uint), cudaMemcpyDeviceToHost), where);
    if (h)
        throw std::runtime_error(std::string(where) + ": index map entries out of range");
}

static void check_dev(bool gpu_contig, const char *where, const char *name)
{
    if (!gpu_contig)
        throw std::runtime_error(std::string(where) + ": '" + name + "' must be a contiguous device array");
}

void get_border_means(Array<float> &out, const Array<float> &signal, const Array<int> &index_map)
{
    const char *where = "get_border_means";
    check_dev(out.gpu && out.is_fully_contiguous(), where, "out");
    check_dev(signal.gpu && signal.is_fully_contiguous(), where, "signal");
    check_dev(index_map.gpu && index_map.is_fully_contiguous(), where, "index_map");
    GMM_ASSERT(out.ndim == 2 && out.shape[1] == 2 && signal.ndim == 2, where);
    GMM_ASSERT(index_map.ndim == 2 && index_map.shape[1] == 5 && index_map.shape[0] == out.shape[0], where);
    Array<uint> w = Array<uint>::alloc_gpu({1}, true);
    throw_on_error(gmm_get_border_means(out.data, signal.data, signal.shape[0], signal.shape[1], index_map.data,
                                        out.shape[0], (uint32_t *) w.data, 0));
    check_range_word(w, where);
}

void deglitch(Array<float> &signal, const Array<float> &bvals, const Array<int> &index_map2)
{
    const char *where = "deglitch";
    check_dev(signal.gpu && signal.is_fully_contiguous(), where, "signal");
    check_dev(bvals.gpu && bvals.is_fully_contiguous(), where, "bvals");
    check_dev(index_map2.gpu && index_map2.is_fully_contiguous(), where, "index_map2");
    GMM_ASSERT(signal.ndim == 2 && bvals.ndim == 2 && bvals.shape[1] == 2, where);
    GMM_ASSERT(index_map2.ndim == 2 && index_map2.shape[1] == 4 && index_map2.shape[0] == bvals.shape[0], where);
    Array<float> cumj = Array<float>::alloc_gpu({std::max<long>(bvals.shape[0], 1)});
    Array<uint> w = Array<uint>::alloc_gpu({1}, true);
    throw_on_error(gmm_deglitch(signal.data, signal.shape[0], signal.shape[1], bvals.data, index_map2.data,
                                bvals.shape[0], cumj.data, (uint32_t *) w.data, 0));
    check_range_word(w, where);
}

void deglitch(Array<float> &signal, const Array<float> &bvals, const Array<float> &cumj, const Array<int> &index_map2)
{
    const char *where = "deglitch";
    check_dev(signal.gpu && signal.is_fully_contiguous(), where, "signal");
    check_dev(bvals.gpu && bvals.is_fully_contiguous(), where, "bvals");
    check_dev(cumj.gpu && cumj.is_fully_contiguous(), where, "cumj");
    check_dev(index_map2.gpu && index_map2.is_fully_contiguous(), where, "index_map2");
    GMM_ASSERT(signal.ndim == 2 && bvals.ndim == 2 && bvals.shape[1] == 2 && cumj.ndim == 1, where);
    GMM_ASSERT(cumj.shape[0] == bvals.shape[0], where);
    GMM_ASSERT(index_map2.ndim == 2 && index_map2.shape[1] == 4 && index_map2.shape[0] == bvals.shape[0], where);
    Array<uint> w = Array<uint>::alloc_gpu({1}, true);
    throw_on_error(gmm_deglitch_cumj(signal.data, signal.shape[0], signal.shape[1], bvals.data, cumj.data,
                                     index_map2.data, bvals.shape[0], (uint32_t *) w.data, 0));
    check_range_word(w, where);
}

void tod_ranges(int mode, Array<float> &tod, Array<float> &rdata, const Array<int> &ostart, const Array<int> &det,
                const Array<int> &istart, const Array<int> &len)
{
    const char *where = (mode == 0) ? "extract_ranges" : (mode == 1) ? "insert_ranges" : "clear_ranges";
    check_dev(tod.gpu && tod.is_fully_contiguous() && tod.ndim == 2, where, "tod");
    check_dev(det.gpu && istart.gpu && len.gpu, where, "dets/starts/lens");
    GMM_ASSERT(det.size == istart.size && det.size == len.size, where);
    if (mode != 2) {
        check_dev(rdata.gpu && rdata.is_fully_contiguous(), where, "junk");
        check_dev(ostart.gpu && ostart.size == det.size, where, "offs");
    }
    Array<uint> w = Array<uint>::alloc_gpu({1}, true);
    int rc;
    if (mode == 0)
        rc = gmm_extract_ranges(tod.data, tod.shape[0], tod.shape[1], rdata.data, rdata.size, ostart.data, det.data,
                                istart.data, len.data, det.size, (uint32_t *) w.data, 0);
    else if (mode == 1)
        rc = gmm_insert_ranges(tod.data, tod.shape[0], tod.shape[1], rdata.data, rdata.size, ostart.data, det.data,
                               istart.data, len.data, det.size, (uint32_t *) w.data, 0);
    else
        rc = gmm_clear_ranges(tod.data, tod.shape[0], tod.shape[1], det.data, istart.data, len.data, det.size,
                              (uint32_t *) w.data, 0);
    throw_on_error(rc);
    check_range_word(w, where);
}

void clip(Array<float> &arr, float vmin, float vmax)
{
    check_dev(arr.gpu && arr.is_fully_contiguous(), "clip", "arr");
    throw_on_error(gmm_clip(arr.data, arr.size, vmin, vmax, 0));
    cuda_check(cudaStreamSynchronize(0), "clip");
}

// ------------------------------------------------------------------------------------------------

#define GMM_INSTANTIATE_PLAN(T)                                                                                   \
    template PointingPrePlan::PointingPrePlan(const Array<T> &, long, long, bool, bool);                         \
    template PointingPrePlan::PointingPrePlan(const Array<T> &, long, long, const Array<uint> &,                 \
                                              const Array<uint> &, bool, bool);                                   \
    template PointingPlan::PointingPlan(const PointingPrePlan &, const Array<T> &, const Array<unsigned char> &, \
                                        const Array<unsigned char> &, bool);                                     \
    template PointingPlan::PointingPlan(const PointingPrePlan &, const Array<T> &, bool);

GMM_INSTANTIATE_PLAN(float)

template void launch_planned_map2tod<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                            const LocalPixelization &, const PointingPlan &, bool, bool, bool);
template void launch_planned_tod2map<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                            const LocalPixelization &, const PointingPlan &, bool, bool);
template void launch_response_map2tod<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                             const Array<float> &, const LocalPixelization &, const PointingPlan &,
                                             bool, bool, bool);
template void launch_response_tod2map<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                             const Array<float> &, const LocalPixelization &, const PointingPlan &,
                                             bool, bool);
template void launch_unplanned_map2tod<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                              const LocalPixelization &, Array<uint> &, bool, bool);
template void launch_unplanned_tod2map<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                              const LocalPixelization &, Array<uint> &, bool);
// Double: the unplanned operators run (f64_kernels.cu); the planned and response ones raise, as the
// reference's cannot launch.
template void launch_planned_map2tod<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                             const LocalPixelization &, const PointingPlan &, bool, bool, bool);
template void launch_planned_tod2map<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                             const LocalPixelization &, const PointingPlan &, bool, bool);
template void launch_response_map2tod<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                              const Array<double> &, const LocalPixelization &, const PointingPlan &,
                                              bool, bool, bool);
template void launch_response_tod2map<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                              const Array<double> &, const LocalPixelization &, const PointingPlan &,
                                              bool, bool);
template void launch_unplanned_map2tod<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                               const LocalPixelization &, Array<uint> &, bool, bool);
template void launch_unplanned_tod2map<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                               const LocalPixelization &, Array<uint> &, bool);
template void reference_map2tod<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                       const LocalPixelization &, bool, bool);
template void reference_map2tod<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                        const LocalPixelization &, bool, bool);
template void reference_tod2map<float>(Array<float> &, const Array<float> &, const Array<float> &,
                                       const LocalPixelization &, bool);
template void reference_tod2map<double>(Array<double> &, const Array<double> &, const Array<double> &,
                                        const LocalPixelization &, bool);
template void local_map_to_global<float>(const LocalPixelization &, Array<float> &, const Array<float> &);
template void local_map_to_global<double>(const LocalPixelization &, Array<double> &, const Array<double> &);
template void check_tod_and_init_nsamp<float>(const Array<float> &, long &, const char *, bool);
template void check_xpointing_and_init_nsamp<float>(const Array<float> &, long &, const char *, bool);
template void check_local_map<float>(const Array<float> &, const LocalPixelization &, const char *, bool);

}  // namespace gpu_mm
