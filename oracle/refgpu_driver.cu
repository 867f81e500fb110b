// Reference-built comparator (TEST INFRASTRUCTURE ONLY).
//
// oracle/Makefile compiles the reference's own plan and operator sources (src_lib/PointingPrePlan.cu,
// PointingPlan.cu, PointingPlanTester.cu, map2tod.cu, tod2map.cu, map2tod_unplanned.cu,
// tod2map_unplanned.cu, map2tod_reference.cu, tod2map_reference.cu, LocalPixelization.cu,
// check_arguments.cu), unchanged and from the reference source tree, together with this file and a
// minimal stand-in for the ksgpu containers they use (oracle/ksgpu_shim), into
// oracle/_ref/libgpu_mm_refgpu.so.  This file only wraps the reference's C++ API
// (include/gpu_mm.hpp:17-247) in extern "C" functions taking raw pointers, for ctypes.
//
// Used by tests (the reference's own PointingPlan / PointingPlanTester as the pin of this
// implementation's plans) and by bench.py (the reference's GPU kernels timed on the same B200).
// Everything runs on the legacy default stream and is synchronous, as in the reference.

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "gpu_mm.hpp"

using namespace gpu_mm;
using ksgpu::Array;

namespace {

thread_local std::string g_err;

// A plan built by the reference's allocating constructors (PointingPrePlan.cu:113-127,
// PointingPlan.cu:316-323).
struct RefPlan {
    PointingPrePlan pp;
    PointingPlan plan;
    RefPlan(const Array<float> &xp, long ny, long nx, bool periodic) :
        pp(xp, ny, nx, periodic), plan(pp, xp) { }
};

// xpointing (3, nsamp) on the GPU.
Array<float> xp_view(const float *xp, long nsamp)
{
    return Array<float>::view(const_cast<float *>(xp), {3, nsamp}, ksgpu::af_gpu);
}

// LocalPixelization from host and device copies of the same cell_offsets (gpu_mm.hpp:30-35).
LocalPixelization make_lpix(long ny, long nx, const long *offs_host, const long *offs_gpu, long nycells, long nxcells,
                            long ystride, long polstride, bool periodic)
{
    Array<long> c = Array<long>::view(const_cast<long *>(offs_host), {nycells, nxcells}, ksgpu::af_uhost);
    Array<long> g = Array<long>::view(const_cast<long *>(offs_gpu), {nycells, nxcells}, ksgpu::af_gpu);
    return LocalPixelization(ny, nx, c, g, ystride, polstride, periodic);
}

template<typename F>
int guarded(F f)
{
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char *refgpu_last_error(void) { return g_err.c_str(); }

// PointingPrePlan + PointingPlan of xpointing (3, nsamp).  Returns a handle, or null (see
// refgpu_last_error()).
void *refgpu_plan_create(const float *xp_gpu, long nsamp, long ny, long nx, int periodic)
{
    RefPlan *p = nullptr;
    int rc = guarded([&] { p = new RefPlan(xp_view(xp_gpu, nsamp), ny, nx, periodic != 0); });
    return rc ? nullptr : p;
}

void refgpu_plan_free(void *h) { delete (RefPlan *) h; }

// info[0..8) = plan_nmt, ncl_per_threadblock, planner_nblocks, nmt_per_threadblock, pointing_nblocks,
// plan_nbytes, plan_constructor_tmp_nbytes, cub_nbytes; overhead separately.
int refgpu_plan_info(void *h, long *info, double *overhead)
{
    const PointingPrePlan &pp = ((RefPlan *) h)->pp;
    info[0] = pp.plan_nmt;
    info[1] = pp.ncl_per_threadblock;
    info[2] = pp.planner_nblocks;
    info[3] = pp.nmt_per_threadblock;
    info[4] = pp.pointing_nblocks;
    info[5] = pp.plan_nbytes;
    info[6] = pp.plan_constructor_tmp_nbytes;
    info[7] = (long) pp.cub_nbytes;
    *overhead = pp.overhead;
    return 0;
}

// Copies plan_mt (plan_nmt words, in the reference's order) and nmt_cumsum (planner_nblocks words)
// to host memory.
int refgpu_plan_get(void *h, uint64_t *mt_host, uint32_t *nmt_cumsum_host)
{
    RefPlan *p = (RefPlan *) h;
    return guarded([&] {
        Array<ulong> mt = p->plan.get_plan_mt(false);
        std::memcpy(mt_host, mt.data, mt.size * sizeof(ulong));
        Array<uint> cs = p->pp.get_nmt_cumsum();
        std::memcpy(nmt_cumsum_host, cs.data, cs.size * sizeof(uint));
    });
}

// PointingPlanTester (PointingPlanTester.cu:69-161): the reference's CPU-side simple plan.  The caller
// passes capacity for plan_nmt words and GMM-preplan-size cumsum words; *nmt receives plan_nmt.
int refgpu_plan_tester(const float *xp_gpu, long nsamp, long ny, long nx, int periodic, uint64_t *sorted_mt_host,
                       long capacity, uint32_t *nmt_cumsum_host, long *nmt)
{
    return guarded([&] {
        Array<float> xp = xp_view(xp_gpu, nsamp);
        PointingPrePlan pp(xp, ny, nx, periodic != 0);
        PointingPlanTester t(pp, xp);
        *nmt = t.plan_nmt;
        if (t.plan_nmt > capacity)
            throw std::runtime_error("refgpu_plan_tester: output capacity too small");
        std::memcpy(sorted_mt_host, t.sorted_mt.data, t.plan_nmt * sizeof(ulong));
        std::memcpy(nmt_cumsum_host, t.nmt_cumsum.data, t.planner_nblocks * sizeof(uint));
    });
}

// launch_planned_map2tod<float> (map2tod.cu:194-272).  tod: nsamp floats; lmap: 3 * npix floats.
int refgpu_planned_map2tod(void *h, float *tod, const float *lmap, long lmap_size, const float *xp, long nsamp,
                           long ny, long nx, const long *offs_host, const long *offs_gpu, long nycells, long nxcells,
                           long ystride, long polstride, int periodic, int partial, int accum)
{
    RefPlan *p = (RefPlan *) h;
    return guarded([&] {
        LocalPixelization lp = make_lpix(ny, nx, offs_host, offs_gpu, nycells, nxcells, ystride, polstride, periodic);
        Array<float> t = Array<float>::view(tod, {nsamp}, ksgpu::af_gpu);
        Array<float> m = Array<float>::view(const_cast<float *>(lmap), {lmap_size}, ksgpu::af_gpu);
        launch_planned_map2tod(t, m, xp_view(xp, nsamp), lp, p->plan, partial != 0, false, accum != 0);
    });
}

// launch_planned_tod2map<float> (tod2map.cu:157-226).  Accumulates into lmap.
int refgpu_planned_tod2map(void *h, float *lmap, long lmap_size, const float *tod, const float *xp, long nsamp,
                           long ny, long nx, const long *offs_host, const long *offs_gpu, long nycells, long nxcells,
                           long ystride, long polstride, int periodic, int partial)
{
    RefPlan *p = (RefPlan *) h;
    return guarded([&] {
        LocalPixelization lp = make_lpix(ny, nx, offs_host, offs_gpu, nycells, nxcells, ystride, polstride, periodic);
        Array<float> m = Array<float>::view(lmap, {lmap_size}, ksgpu::af_gpu);
        Array<float> t = Array<float>::view(const_cast<float *>(tod), {nsamp}, ksgpu::af_gpu);
        launch_planned_tod2map(m, t, xp_view(xp, nsamp), lp, p->plan, partial != 0, false);
    });
}

// launch_unplanned_map2tod<float> / launch_unplanned_tod2map<float> (map2tod_unplanned.cu:75-127,
// tod2map_unplanned.cu:70-121) with 'errflags' of nerr words on the GPU (the Python wrapper uses 2048).
int refgpu_unplanned_map2tod(float *tod, const float *lmap, long lmap_size, const float *xp, long nsamp, long ny,
                             long nx, const long *offs_host, const long *offs_gpu, long nycells, long nxcells,
                             long ystride, long polstride, int periodic, uint32_t *errflags_gpu, long nerr,
                             int partial, int accum)
{
    return guarded([&] {
        LocalPixelization lp = make_lpix(ny, nx, offs_host, offs_gpu, nycells, nxcells, ystride, polstride, periodic);
        Array<float> t = Array<float>::view(tod, {nsamp}, ksgpu::af_gpu);
        Array<float> m = Array<float>::view(const_cast<float *>(lmap), {lmap_size}, ksgpu::af_gpu);
        Array<uint> e = Array<uint>::view(errflags_gpu, {nerr}, ksgpu::af_gpu);
        launch_unplanned_map2tod(t, m, xp_view(xp, nsamp), lp, e, partial != 0, accum != 0);
    });
}

int refgpu_unplanned_tod2map(float *lmap, long lmap_size, const float *tod, const float *xp, long nsamp, long ny,
                             long nx, const long *offs_host, const long *offs_gpu, long nycells, long nxcells,
                             long ystride, long polstride, int periodic, uint32_t *errflags_gpu, long nerr,
                             int partial)
{
    return guarded([&] {
        LocalPixelization lp = make_lpix(ny, nx, offs_host, offs_gpu, nycells, nxcells, ystride, polstride, periodic);
        Array<float> m = Array<float>::view(lmap, {lmap_size}, ksgpu::af_gpu);
        Array<float> t = Array<float>::view(const_cast<float *>(tod), {nsamp}, ksgpu::af_gpu);
        Array<uint> e = Array<uint>::view(errflags_gpu, {nerr}, ksgpu::af_gpu);
        launch_unplanned_tod2map(m, t, xp_view(xp, nsamp), lp, e, partial != 0);
    });
}

// reference_map2tod<float> / reference_tod2map<float> (map2tod_reference.cu:16-54,
// tod2map_reference.cu:14-46): the reference's single-threaded CPU operators, on host arrays.
int refgpu_reference_map2tod(float *tod, const float *lmap, long lmap_size, const float *xp, long nsamp, long ny,
                             long nx, const long *offs_host, long nycells, long nxcells, long ystride, long polstride,
                             int periodic, int partial, int accum)
{
    return guarded([&] {
        Array<long> c = Array<long>::view(const_cast<long *>(offs_host), {nycells, nxcells}, ksgpu::af_uhost);
        LocalPixelization lp(ny, nx, c, c, ystride, polstride, periodic != 0);
        Array<float> t = Array<float>::view(tod, {nsamp}, ksgpu::af_uhost);
        Array<float> m = Array<float>::view(const_cast<float *>(lmap), {lmap_size}, ksgpu::af_uhost);
        Array<float> x = Array<float>::view(const_cast<float *>(xp), {3, nsamp}, ksgpu::af_uhost);
        reference_map2tod(t, m, x, lp, partial != 0, accum != 0);
    });
}

int refgpu_reference_tod2map(float *lmap, long lmap_size, const float *tod, const float *xp, long nsamp, long ny,
                             long nx, const long *offs_host, long nycells, long nxcells, long ystride, long polstride,
                             int periodic, int partial)
{
    return guarded([&] {
        Array<long> c = Array<long>::view(const_cast<long *>(offs_host), {nycells, nxcells}, ksgpu::af_uhost);
        LocalPixelization lp(ny, nx, c, c, ystride, polstride, periodic != 0);
        Array<float> m = Array<float>::view(lmap, {lmap_size}, ksgpu::af_uhost);
        Array<float> t = Array<float>::view(const_cast<float *>(tod), {nsamp}, ksgpu::af_uhost);
        Array<float> x = Array<float>::view(const_cast<float *>(xp), {3, nsamp}, ksgpu::af_uhost);
        reference_tod2map(m, t, x, lp, partial != 0);
    });
}

}  // extern "C"
