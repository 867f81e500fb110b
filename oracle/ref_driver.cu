// Reference-built checker (TEST INFRASTRUCTURE ONLY).
//
// This file is compiled against the reference's own header include/gpu_mm_internals.hpp, taken
// from the reference source tree at build time (see oracle/Makefile; nothing is copied into this
// repository).  That header holds the reference's complete per-sample arithmetic:
// pixel_locator (gpu_mm_internals.hpp:104-176), cell_enumerator (:179-237), map_evaluator
// (:243-293) and map_accumulator (:299-355).  The 15-line sample loops of map2tod_reference.cu:35-50
// and tod2map_reference.cu:32-43 are restated here around those templates, so that this library
// needs nothing but the header (the reference's .cu files themselves, which need ksgpu, are built
// against a stand-in into libgpu_mm_refgpu.so by refgpu_driver.cu).
//
// Outputs go to oracle/_ref/ only.  Used by tests (as the pin of the C restatement in oracle.c)
// and by bench.py's reference arm (kind "reference": the reference's CPU operator arithmetic).

#include <sys/types.h>
#include <cstdint>
#include <cmath>
#include <pthread.h>
#include <vector>

#include "gpu_mm_internals.hpp"

using namespace gpu_mm;

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
} ref_lpix;

extern "C" uint32_t ref_locate_f32(float ypix, float xpix, int32_t ny, int32_t nx, int32_t periodic,
                        int32_t out_idx[4], float out_d[2])
{
    pixel_locator<float> px(ny, nx, periodic != 0);
    uint err = 0;
    px.locate(ypix, xpix, err);
    out_idx[0] = px.iy0; out_idx[1] = px.iy1; out_idx[2] = px.ix0; out_idx[3] = px.ix1;
    out_d[0] = px.dy; out_d[1] = px.dx;
    return err;
}

template<typename T>
static uint32_t map2tod_range(T *tod, const T *lmap, const T *xp, int64_t nsamp, int64_t s0, int64_t s1,
                              const ref_lpix *lp, int partial, int accum)
{
    map_evaluator<T,false> mev(lmap, (const long *) lp->cell_offsets, lp->nycells, lp->nxcells,
                               lp->ystride, lp->polstride, partial != 0);
    pixel_locator<T> px(lp->nypix_global, lp->nxpix_global, lp->periodic_xcoord != 0);
    uint err = 0;
    for (long s = s0; s < s1; s++) {
        T ypix = xp[s];
        T xpix = xp[s + nsamp];
        T alpha = xp[s + 2*nsamp];
        T sin_2a, cos_2a;
        dtype<T>::xsincos(2*alpha, &sin_2a, &cos_2a);
        px.locate(ypix, xpix, err);
        T t = mev.eval(px, cos_2a, sin_2a, err);
        if (accum)
            tod[s] += t;
        else
            tod[s] = t;
    }
    return err;
}

template<typename T>
static uint32_t tod2map_range(T *lmap, const T *tod, const T *xp, int64_t nsamp, int64_t s0, int64_t s1,
                              const ref_lpix *lp, int partial)
{
    map_accumulator<T,false> macc(lmap, (const long *) lp->cell_offsets, lp->nycells, lp->nxcells,
                                  lp->ystride, lp->polstride, partial != 0);
    pixel_locator<T> px(lp->nypix_global, lp->nxpix_global, lp->periodic_xcoord != 0);
    uint err = 0;
    for (long s = s0; s < s1; s++) {
        T ypix = xp[s];
        T xpix = xp[s + nsamp];
        T alpha = xp[s + 2*nsamp];
        T t = tod[s];
        T sin_2a, cos_2a;
        dtype<T>::xsincos(2*alpha, &sin_2a, &cos_2a);
        px.locate(ypix, xpix, err);
        macc.accum(px, t, t*cos_2a, t*sin_2a, err);
    }
    return err;
}

extern "C" uint32_t ref_map2tod_f32(float *tod, const float *lmap, const float *xp, int64_t nsamp,
                         const ref_lpix *lp, int32_t partial, int32_t accum)
{ return map2tod_range<float>(tod, lmap, xp, nsamp, 0, nsamp, lp, partial, accum); }

extern "C" uint32_t ref_map2tod_f64(double *tod, const double *lmap, const double *xp, int64_t nsamp,
                         const ref_lpix *lp, int32_t partial, int32_t accum)
{ return map2tod_range<double>(tod, lmap, xp, nsamp, 0, nsamp, lp, partial, accum); }

extern "C" uint32_t ref_tod2map_f32(float *lmap, const float *tod, const float *xp, int64_t nsamp,
                         const ref_lpix *lp, int32_t partial)
{ return tod2map_range<float>(lmap, tod, xp, nsamp, 0, nsamp, lp, partial); }

extern "C" uint32_t ref_tod2map_f64(double *lmap, const double *tod, const double *xp, int64_t nsamp,
                         const ref_lpix *lp, int32_t partial)
{ return tod2map_range<double>(lmap, tod, xp, nsamp, 0, nsamp, lp, partial); }

// Multi-threaded timing driver: contiguous sample ranges per thread; tod2map uses a private map
// per thread followed by a sum (the reference's CPU operators are single-threaded by design).
struct ref_job {
    float *out; const float *lmap; const float *tod; const float *xp;
    int64_t nsamp, s0, s1; const ref_lpix *lp; int partial, accum; uint32_t err;
};

static void *ref_m2t_worker(void *a)
{
    ref_job *j = (ref_job *) a;
    j->err = map2tod_range<float>(j->out, j->lmap, j->xp, j->nsamp, j->s0, j->s1, j->lp, j->partial, j->accum);
    return nullptr;
}

static void *ref_t2m_worker(void *a)
{
    ref_job *j = (ref_job *) a;
    j->err = tod2map_range<float>(j->out, j->tod, j->xp, j->nsamp, j->s0, j->s1, j->lp, j->partial);
    return nullptr;
}

extern "C" uint32_t ref_map2tod_f32_mt(float *tod, const float *lmap, const float *xp, int64_t nsamp,
                            const ref_lpix *lp, int32_t partial, int32_t accum, int32_t nthreads)
{
    if (nthreads < 1) nthreads = 1;
    std::vector<pthread_t> th(nthreads);
    std::vector<ref_job> jobs(nthreads);
    for (int i = 0; i < nthreads; i++) {
        jobs[i] = ref_job{tod, lmap, nullptr, xp, nsamp, nsamp*i/nthreads, nsamp*(i+1)/nthreads, lp, partial, accum, 0};
        pthread_create(&th[i], nullptr, ref_m2t_worker, &jobs[i]);
    }
    uint32_t err = 0;
    for (int i = 0; i < nthreads; i++) { pthread_join(th[i], nullptr); err |= jobs[i].err; }
    return err;
}

extern "C" uint32_t ref_tod2map_f32_mt(float *lmap, const float *tod, const float *xp, int64_t nsamp, int64_t map_size,
                            const ref_lpix *lp, int32_t partial, int32_t nthreads)
{
    if (nthreads < 1) nthreads = 1;
    std::vector<pthread_t> th(nthreads);
    std::vector<ref_job> jobs(nthreads);
    std::vector<std::vector<float>> priv(nthreads);
    for (int i = 0; i < nthreads; i++) {
        priv[i].assign(map_size, 0.0f);
        jobs[i] = ref_job{priv[i].data(), nullptr, tod, xp, nsamp, nsamp*i/nthreads, nsamp*(i+1)/nthreads, lp, partial, 0, 0};
        pthread_create(&th[i], nullptr, ref_t2m_worker, &jobs[i]);
    }
    uint32_t err = 0;
    for (int i = 0; i < nthreads; i++) { pthread_join(th[i], nullptr); err |= jobs[i].err; }
    for (int i = 0; i < nthreads; i++)
        for (int64_t k = 0; k < map_size; k++)
            lmap[k] += priv[i][k];
    return err;
}

// The reference's cell_enumerator is device-only; this kernel runs it on the GPU so that the
// oracle's restatement of the cell slots can be checked against the reference's own code.
__global__ void ref_enumerate_kernel(const float *xp, long nsamp, int ny, int nx, bool periodic,
                                     int *slots, uint *errs)
{
    long s = blockIdx.x * long(blockDim.x) + threadIdx.x;
    if (s >= nsamp)
        return;
    cell_enumerator<float,false> cells(ny, nx, periodic);
    uint err = 0;
    cells.enumerate(xp[s], xp[s + nsamp], err);
    int iy[2] = {cells.iy0, cells.iy1};
    int ix[3] = {cells.ix0, cells.ix1, cells.ix2};
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 3; b++)
            slots[6*s + 3*a + b] = ((iy[a] >= 0) && (ix[b] >= 0)) ? ((iy[a] << 10) | ix[b]) : -1;
    errs[s] = err;
}

extern "C" int32_t ref_enumerate_gpu(const float *xp_dev, int64_t nsamp, int32_t ny, int32_t nx,
                                     int32_t periodic, int32_t *slots_dev, uint32_t *errs_dev)
{
    int threads = 128;
    long blocks = (nsamp + threads - 1) / threads;
    ref_enumerate_kernel<<<blocks, threads>>>(xp_dev, nsamp, ny, nx, periodic != 0, slots_dev, errs_dev);
    cudaError_t e = cudaDeviceSynchronize();
    return (int32_t) e;
}
