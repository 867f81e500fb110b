/*
 * CPU oracle for the gpu_mm pointing-operator hot path (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Compiled with -ffp-contract=off so that float expressions are evaluated exactly as written,
 * like the reference's host build of map2tod_reference.cu / tod2map_reference.cu.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* pixel_locator (gpu_mm_internals.hpp:124-164)                                                */

#define DEFINE_LOCATE(T, SUFFIX)                                                                \
    static inline uint32_t locate_##SUFFIX(T ypix, T xpix, int ny, int nx, int periodic,       \
                                           int *iy0, int *iy1, int *ix0, int *ix1,             \
                                           T *dy, T *dx)                                       \
    {                                                                                          \
        uint32_t err = 0;                                                                      \
        int y0 = (int) ypix;                                                                   \
        y0 = (y0 > 0) ? y0 : 0;                                                                \
        y0 = (y0 < ny - 2) ? y0 : (ny - 2);                                                    \
        *iy0 = y0;                                                                             \
        *iy1 = y0 + 1;                                                                         \
        *dy = ypix - (T) y0;                                                                   \
        if (!((ypix >= 0) && (ypix <= (T) (ny - 1))))                                          \
            err |= ORACLE_ERR_BAD_YPIX;                                                        \
        if (periodic) {                                                                        \
            if (!((xpix >= (T) (-nx)) && (xpix <= (T) (2 * nx))))                              \
                err |= ORACLE_ERR_BAD_XPIX;                                                    \
            xpix = (xpix >= 0) ? xpix : (xpix + (T) nx);                                       \
            xpix = (xpix <= (T) nx) ? xpix : (xpix - (T) nx);                                  \
            int x0 = (int) xpix;                                                               \
            x0 = (x0 > 0) ? x0 : 0;                                                            \
            *dx = xpix - (T) x0;                                                               \
            x0 = (x0 < nx) ? x0 : 0;                                                           \
            int x1 = x0 + 1;                                                                   \
            x1 = (x1 < nx) ? x1 : 0;                                                           \
            *ix0 = x0;                                                                         \
            *ix1 = x1;                                                                         \
        } else {                                                                               \
            if (!((xpix >= 0) && (xpix <= (T) (nx - 2))))                                      \
                err |= ORACLE_ERR_BAD_XPIX;                                                    \
            int x0 = (int) xpix;                                                               \
            x0 = (x0 > 0) ? x0 : 0;                                                            \
            x0 = (x0 < nx - 2) ? x0 : (nx - 2);                                                \
            *ix0 = x0;                                                                         \
            *ix1 = x0 + 1;                                                                     \
            *dx = xpix - (T) x0;                                                               \
        }                                                                                      \
        return err;                                                                            \
    }

/* float -> int conversion of NaN/huge values is undefined in C; the reference only relies on the
 * error bit in those cases (the clamped indices stay in range), so clamp the input first. */
static inline float sanitize_f32(float v) { return (v == v) ? fminf(fmaxf(v, -2.0e9f), 2.0e9f) : -1.0f; }
static inline double sanitize_f64(double v) { return (v == v) ? fmin(fmax(v, -2.0e9), 2.0e9) : -1.0; }

DEFINE_LOCATE(float, raw_f32)
DEFINE_LOCATE(double, raw_f64)

static inline uint32_t locate_f32(float ypix, float xpix, int ny, int nx, int periodic,
                                  int *iy0, int *iy1, int *ix0, int *ix1, float *dy, float *dx)
{
    uint32_t e = 0;
    if (!(ypix == ypix)) e |= ORACLE_ERR_BAD_YPIX;
    if (!(xpix == xpix)) e |= ORACLE_ERR_BAD_XPIX;
    return e | locate_raw_f32(sanitize_f32(ypix), sanitize_f32(xpix), ny, nx, periodic, iy0, iy1, ix0, ix1, dy, dx);
}

static inline uint32_t locate_f64(double ypix, double xpix, int ny, int nx, int periodic,
                                  int *iy0, int *iy1, int *ix0, int *ix1, double *dy, double *dx)
{
    uint32_t e = 0;
    if (!(ypix == ypix)) e |= ORACLE_ERR_BAD_YPIX;
    if (!(xpix == xpix)) e |= ORACLE_ERR_BAD_XPIX;
    return e | locate_raw_f64(sanitize_f64(ypix), sanitize_f64(xpix), ny, nx, periodic, iy0, iy1, ix0, ix1, dy, dx);
}

uint32_t oracle_locate_f32(float ypix, float xpix, int32_t ny, int32_t nx, int32_t periodic,
                           int32_t out_idx[4], float out_d[2])
{
    int iy0, iy1, ix0, ix1;
    float dy, dx;
    uint32_t err = locate_f32(ypix, xpix, ny, nx, periodic, &iy0, &iy1, &ix0, &ix1, &dy, &dx);
    out_idx[0] = iy0; out_idx[1] = iy1; out_idx[2] = ix0; out_idx[3] = ix1;
    out_d[0] = dy; out_d[1] = dx;
    return err;
}

uint32_t oracle_locate_f64(double ypix, double xpix, int32_t ny, int32_t nx, int32_t periodic,
                           int32_t out_idx[4], double out_d[2])
{
    int iy0, iy1, ix0, ix1;
    double dy, dx;
    uint32_t err = locate_f64(ypix, xpix, ny, nx, periodic, &iy0, &iy1, &ix0, &ix1, &dy, &dx);
    out_idx[0] = iy0; out_idx[1] = iy1; out_idx[2] = ix0; out_idx[3] = ix1;
    out_d[0] = dy; out_d[1] = dx;
    return err;
}

/* ------------------------------------------------------------------------------------------ */
/* map_evaluator / map_accumulator (gpu_mm_internals.hpp:243-355)                              */

static inline int64_t pixel_offset(const oracle_lpix *lp, int iy, int ix)
{
    int iyc = iy >> 6, ixc = ix >> 6;
    int valid = (iy >= 0) && (ix >= 0) && (iyc < lp->nycells) && (ixc < lp->nxcells);
    int64_t off = valid ? lp->cell_offsets[(int64_t) iyc * lp->nxcells + ixc] : -1;
    if (off < 0)
        return -1;
    return off + (ix - (ixc << 6)) + (int64_t) (iy - (iyc << 6)) * lp->ystride;
}

#define DEFINE_OPS(T, SUFFIX, SINCOS)                                                          \
    static inline T eval_##SUFFIX(const T *lmap, const oracle_lpix *lp, int iy, int ix,       \
                                  T c, T s, int partial, uint32_t *err)                        \
    {                                                                                          \
        int64_t off = pixel_offset(lp, iy, ix);                                                \
        int valid = (off >= 0);                                                                \
        T t = valid ? lmap[off] : 0;                                                           \
        T q = valid ? lmap[off + lp->polstride] : 0;                                           \
        T u = valid ? lmap[off + 2 * lp->polstride] : 0;                                       \
        if (!(valid || partial)) *err |= ORACLE_ERR_NOT_IN_PIXELIZATION;                       \
        return t + c * q + s * u;                                                              \
    }                                                                                          \
    static inline void accum_##SUFFIX(T *lmap, const oracle_lpix *lp, int iy, int ix,          \
                                      T t, T q, T u, T w, int partial, uint32_t *err)          \
    {                                                                                          \
        int64_t off = pixel_offset(lp, iy, ix);                                                \
        int valid = (off >= 0);                                                                \
        if (valid) {                                                                           \
            lmap[off] += w * t;                                                                \
            lmap[off + lp->polstride] += w * q;                                                \
            lmap[off + 2 * lp->polstride] += w * u;                                            \
        }                                                                                      \
        if (!(valid || partial)) *err |= ORACLE_ERR_NOT_IN_PIXELIZATION;                       \
    }                                                                                          \
    /* map2tod_reference.cu:35-50 */                                                           \
    static uint32_t map2tod_range_##SUFFIX(T *tod, const T *lmap, const T *xp, int64_t nsamp,  \
                                           int64_t s0, int64_t s1, const oracle_lpix *lp,      \
                                           int partial, int accum)                             \
    {                                                                                          \
        uint32_t err = 0;                                                                      \
        for (int64_t s = s0; s < s1; s++) {                                                    \
            T ypix = xp[s], xpix = xp[s + nsamp], alpha = xp[s + 2 * nsamp];                  \
            T sn, cs;                                                                          \
            SINCOS(2 * alpha, &sn, &cs);                                                       \
            int iy0, iy1, ix0, ix1;                                                            \
            T dy, dx;                                                                          \
            err |= locate_##SUFFIX(ypix, xpix, lp->nypix_global, lp->nxpix_global,             \
                                   lp->periodic_xcoord, &iy0, &iy1, &ix0, &ix1, &dy, &dx);     \
            T r = (1 - dy) * (1 - dx) * eval_##SUFFIX(lmap, lp, iy0, ix0, cs, sn, partial, &err); \
            r += (1 - dy) * (dx) * eval_##SUFFIX(lmap, lp, iy0, ix1, cs, sn, partial, &err);   \
            r += (dy) * (1 - dx) * eval_##SUFFIX(lmap, lp, iy1, ix0, cs, sn, partial, &err);   \
            r += (dy) * (dx) * eval_##SUFFIX(lmap, lp, iy1, ix1, cs, sn, partial, &err);       \
            if (accum) tod[s] += r; else tod[s] = r;                                           \
        }                                                                                      \
        return err;                                                                            \
    }                                                                                          \
    /* tod2map_reference.cu:32-43 */                                                           \
    static uint32_t tod2map_range_##SUFFIX(T *lmap, const T *tod, const T *xp, int64_t nsamp,  \
                                           int64_t s0, int64_t s1, const oracle_lpix *lp,      \
                                           int partial)                                        \
    {                                                                                          \
        uint32_t err = 0;                                                                      \
        for (int64_t s = s0; s < s1; s++) {                                                    \
            T ypix = xp[s], xpix = xp[s + nsamp], alpha = xp[s + 2 * nsamp];                  \
            T t = tod[s];                                                                      \
            T sn, cs;                                                                          \
            SINCOS(2 * alpha, &sn, &cs);                                                       \
            int iy0, iy1, ix0, ix1;                                                            \
            T dy, dx;                                                                          \
            err |= locate_##SUFFIX(ypix, xpix, lp->nypix_global, lp->nxpix_global,             \
                                   lp->periodic_xcoord, &iy0, &iy1, &ix0, &ix1, &dy, &dx);     \
            T q = t * cs, u = t * sn;                                                          \
            accum_##SUFFIX(lmap, lp, iy0, ix0, t, q, u, (1 - dy) * (1 - dx), partial, &err);   \
            accum_##SUFFIX(lmap, lp, iy0, ix1, t, q, u, (1 - dy) * (dx), partial, &err);       \
            accum_##SUFFIX(lmap, lp, iy1, ix0, t, q, u, (dy) * (1 - dx), partial, &err);       \
            accum_##SUFFIX(lmap, lp, iy1, ix1, t, q, u, (dy) * (dx), partial, &err);           \
        }                                                                                      \
        return err;                                                                            \
    }

DEFINE_OPS(float, f32, sincosf)
DEFINE_OPS(double, f64, sincos)

uint32_t oracle_map2tod_f32(float *tod, const float *lmap, const float *xp, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial, int32_t accum)
{
    return map2tod_range_f32(tod, lmap, xp, nsamp, 0, nsamp, lp, partial, accum);
}

uint32_t oracle_map2tod_f64(double *tod, const double *lmap, const double *xp, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial, int32_t accum)
{
    return map2tod_range_f64(tod, lmap, xp, nsamp, 0, nsamp, lp, partial, accum);
}

uint32_t oracle_tod2map_f32(float *lmap, const float *tod, const float *xp, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial)
{
    return tod2map_range_f32(lmap, tod, xp, nsamp, 0, nsamp, lp, partial);
}

uint32_t oracle_tod2map_f64(double *lmap, const double *tod, const double *xp, int64_t nsamp,
                            const oracle_lpix *lp, int32_t partial)
{
    return tod2map_range_f64(lmap, tod, xp, nsamp, 0, nsamp, lp, partial);
}

uint32_t oracle_map2tod_f32_range(float *tod, const float *lmap, const float *xp, int64_t nsamp,
                                  int64_t s0, int64_t s1, const oracle_lpix *lp, int32_t partial, int32_t accum)
{
    return map2tod_range_f32(tod, lmap, xp, nsamp, s0, s1, lp, partial, accum);
}

uint32_t oracle_tod2map_f32_range(float *lmap, const float *tod, const float *xp, int64_t nsamp,
                                  int64_t s0, int64_t s1, const oracle_lpix *lp, int32_t partial)
{
    return tod2map_range_f32(lmap, tod, xp, nsamp, s0, s1, lp, partial);
}

/* Response variants: map2tod_response.cu:164-193 and tod2map_response.cu:104-124. */
uint32_t oracle_response_map2tod_f32(float *tod, const float *lmap, const float *xp, const float *resp,
                                     int64_t ndet, int64_t nperdet, const oracle_lpix *lp,
                                     int32_t partial, int32_t accum)
{
    int64_t nsamp = ndet * nperdet;
    uint32_t err = 0;
    for (int64_t s = 0; s < nsamp; s++) {
        float ypix = xp[s], xpix = xp[s + nsamp], alpha = xp[s + 2 * nsamp];
        int64_t det = s / nperdet;
        float t_resp = resp[det], p_resp = resp[det + ndet];
        float sn, cs;
        sincosf(2 * alpha, &sn, &cs);
        float q_resp = p_resp * cs, u_resp = p_resp * sn;
        int iy0, iy1, ix0, ix1;
        float dy, dx;
        err |= locate_f32(ypix, xpix, lp->nypix_global, lp->nxpix_global, lp->periodic_xcoord,
                          &iy0, &iy1, &ix0, &ix1, &dy, &dx);
        int iys[4] = {iy0, iy0, iy1, iy1}, ixs[4] = {ix0, ix1, ix0, ix1};
        float ws[4] = {(1 - dy) * (1 - dx), (1 - dy) * (dx), (dy) * (1 - dx), (dy) * (dx)};
        float r = 0;
        for (int k = 0; k < 4; k++) {
            int64_t off = pixel_offset(lp, iys[k], ixs[k]);
            int valid = (off >= 0);
            float v = valid ? (t_resp * lmap[off] + q_resp * lmap[off + lp->polstride]
                               + u_resp * lmap[off + 2 * lp->polstride]) : 0.0f;
            if (!(valid || partial)) err |= ORACLE_ERR_NOT_IN_PIXELIZATION;
            r = (k == 0) ? ws[k] * v : (r + ws[k] * v);
        }
        if (accum) tod[s] += r; else tod[s] = r;
    }
    return err;
}

uint32_t oracle_response_tod2map_f32(float *lmap, const float *tod, const float *xp, const float *resp,
                                     int64_t ndet, int64_t nperdet, const oracle_lpix *lp, int32_t partial)
{
    int64_t nsamp = ndet * nperdet;
    uint32_t err = 0;
    for (int64_t s = 0; s < nsamp; s++) {
        float ypix = xp[s], xpix = xp[s + nsamp], alpha = xp[s + 2 * nsamp];
        int64_t det = s / nperdet;
        float t_resp = resp[det], p_resp = resp[det + ndet];
        float sn, cs;
        sincosf(2 * alpha, &sn, &cs);
        float t = t_resp * tod[s];
        float q = p_resp * tod[s] * cs;
        float u = p_resp * tod[s] * sn;
        int iy0, iy1, ix0, ix1;
        float dy, dx;
        err |= locate_f32(ypix, xpix, lp->nypix_global, lp->nxpix_global, lp->periodic_xcoord,
                          &iy0, &iy1, &ix0, &ix1, &dy, &dx);
        accum_f32(lmap, lp, iy0, ix0, t, q, u, (1 - dy) * (1 - dx), partial, &err);
        accum_f32(lmap, lp, iy0, ix1, t, q, u, (1 - dy) * (dx), partial, &err);
        accum_f32(lmap, lp, iy1, ix0, t, q, u, (dy) * (1 - dx), partial, &err);
        accum_f32(lmap, lp, iy1, ix1, t, q, u, (dy) * (dx), partial, &err);
    }
    return err;
}

/* ------------------------------------------------------------------------------------------ */
/* Multi-threaded CPU baseline: contiguous sample ranges per thread.                           */

/* reference_tod2map<double> (tod2map_reference.cu:32-43) on float32 TOD and xpointing widened to
 * double: the FP64 oracle of the tod2map precision variants. */
static uint32_t tod2map_range_f64w(double *lmap, const float *tod, const float *xp, int64_t nsamp, int64_t s0,
                                   int64_t s1, const oracle_lpix *lp, int partial)
{
    uint32_t err = 0;
    for (int64_t s = s0; s < s1; s++) {
        double ypix = xp[s], xpix = xp[s + nsamp], alpha = xp[s + 2 * nsamp];
        double t = tod[s];
        double sn, cs;
        sincos(2 * alpha, &sn, &cs);
        int iy0, iy1, ix0, ix1;
        double dy, dx;
        err |= locate_f64(ypix, xpix, lp->nypix_global, lp->nxpix_global, lp->periodic_xcoord, &iy0, &iy1, &ix0,
                          &ix1, &dy, &dx);
        double q = t * cs, u = t * sn;
        accum_f64(lmap, lp, iy0, ix0, t, q, u, (1 - dy) * (1 - dx), partial, &err);
        accum_f64(lmap, lp, iy0, ix1, t, q, u, (1 - dy) * (dx), partial, &err);
        accum_f64(lmap, lp, iy1, ix0, t, q, u, (dy) * (1 - dx), partial, &err);
        accum_f64(lmap, lp, iy1, ix1, t, q, u, (dy) * (dx), partial, &err);
    }
    return err;
}

typedef struct {
    double *out;
    const float *tod, *xp;
    int64_t nsamp, s0, s1;
    const oracle_lpix *lp;
    int partial;
    uint32_t err;
} mt_job_f64w;

static void *tod2map_f64w_worker(void *arg)
{
    mt_job_f64w *j = (mt_job_f64w *) arg;
    j->err = tod2map_range_f64w(j->out, j->tod, j->xp, j->nsamp, j->s0, j->s1, j->lp, j->partial);
    return NULL;
}

uint32_t oracle_tod2map_f64w_mt(double *lmap, const float *tod, const float *xp, int64_t nsamp, int64_t map_size,
                                const oracle_lpix *lp, int32_t partial, int32_t nthreads)
{
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
    mt_job_f64w *jobs = (mt_job_f64w *) calloc(nthreads, sizeof(mt_job_f64w));
    double **priv = (double **) calloc(nthreads, sizeof(double *));
    for (int i = 0; i < nthreads; i++) {
        priv[i] = (double *) calloc(map_size, sizeof(double));
        jobs[i] = (mt_job_f64w) {priv[i], tod, xp, nsamp, nsamp * i / nthreads, nsamp * (i + 1) / nthreads, lp,
                                 partial, 0};
        pthread_create(&th[i], NULL, tod2map_f64w_worker, &jobs[i]);
    }
    uint32_t err = 0;
    for (int i = 0; i < nthreads; i++) {
        pthread_join(th[i], NULL);
        err |= jobs[i].err;
    }
    for (int i = 0; i < nthreads; i++) {
        for (int64_t k = 0; k < map_size; k++)
            lmap[k] += priv[i][k];
        free(priv[i]);
    }
    free(priv);
    free(th);
    free(jobs);
    return err;
}

typedef struct {
    float *out;
    const float *lmap;
    const float *tod;
    const float *xp;
    int64_t nsamp, s0, s1;
    const oracle_lpix *lp;
    int partial, accum;
    uint32_t err;
} mt_job;

static void *map2tod_worker(void *arg)
{
    mt_job *j = (mt_job *) arg;
    j->err = map2tod_range_f32(j->out, j->lmap, j->xp, j->nsamp, j->s0, j->s1, j->lp, j->partial, j->accum);
    return NULL;
}

static void *tod2map_worker(void *arg)
{
    mt_job *j = (mt_job *) arg;
    j->err = tod2map_range_f32(j->out, j->tod, j->xp, j->nsamp, j->s0, j->s1, j->lp, j->partial);
    return NULL;
}

uint32_t oracle_map2tod_f32_mt(float *tod, const float *lmap, const float *xp, int64_t nsamp,
                               const oracle_lpix *lp, int32_t partial, int32_t accum, int32_t nthreads)
{
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
    mt_job *jobs = (mt_job *) calloc(nthreads, sizeof(mt_job));
    for (int i = 0; i < nthreads; i++) {
        jobs[i] = (mt_job) {tod, lmap, NULL, xp, nsamp, nsamp * i / nthreads, nsamp * (i + 1) / nthreads,
                            lp, partial, accum, 0};
        pthread_create(&th[i], NULL, map2tod_worker, &jobs[i]);
    }
    uint32_t err = 0;
    for (int i = 0; i < nthreads; i++) {
        pthread_join(th[i], NULL);
        err |= jobs[i].err;
    }
    free(th);
    free(jobs);
    return err;
}

uint32_t oracle_tod2map_f32_mt(float *lmap, const float *tod, const float *xp, int64_t nsamp, int64_t map_size,
                               const oracle_lpix *lp, int32_t partial, int32_t nthreads)
{
    if (nthreads < 1) nthreads = 1;
    pthread_t *th = (pthread_t *) calloc(nthreads, sizeof(pthread_t));
    mt_job *jobs = (mt_job *) calloc(nthreads, sizeof(mt_job));
    float **priv = (float **) calloc(nthreads, sizeof(float *));
    for (int i = 0; i < nthreads; i++) {
        priv[i] = (float *) calloc(map_size, sizeof(float));
        jobs[i] = (mt_job) {priv[i], NULL, tod, xp, nsamp, nsamp * i / nthreads, nsamp * (i + 1) / nthreads,
                            lp, partial, 0, 0};
        pthread_create(&th[i], NULL, tod2map_worker, &jobs[i]);
    }
    uint32_t err = 0;
    for (int i = 0; i < nthreads; i++) {
        pthread_join(th[i], NULL);
        err |= jobs[i].err;
    }
    for (int i = 0; i < nthreads; i++) {
        for (int64_t k = 0; k < map_size; k++)
            lmap[k] += priv[i][k];
        free(priv[i]);
    }
    free(priv);
    free(th);
    free(jobs);
    return err;
}

/* ------------------------------------------------------------------------------------------ */
/* Plan oracle.                                                                                */

/* Cell "slots" of one sample, restating cell_enumerator::enumerate (gpu_mm_internals.hpp:194-236):
 * y-slot 0 holds the even y-cell, y-slot 1 the odd one; x-slot 0 the even non-zero x-cell, x-slot 1
 * the odd one, x-slot 2 the x-cell 0.  Absent entries are -1.  Slot k = 3*yslot + xslot, in the
 * order ca0..ca5 of PointingPlan.cu:173-178. */
static inline void sample_slots(int iy0, int iy1, int ix0, int ix1, int slots[6])
{
    int yc[2] = {-1, -1}, xc[3] = {-1, -1, -1};
    int iyc0 = iy0 >> 6, iyc1 = iy1 >> 6, ixc0 = ix0 >> 6, ixc1 = ix1 >> 6;
    yc[iyc0 & 1] = iyc0;
    if (iyc1 != iyc0) yc[iyc1 & 1] = iyc1;
    xc[(ixc0 == 0) ? 2 : (ixc0 & 1)] = ixc0;
    if (ixc1 != ixc0) xc[(ixc1 == 0) ? 2 : (ixc1 & 1)] = ixc1;
    for (int a = 0; a < 2; a++)
        for (int b = 0; b < 3; b++)
            slots[3 * a + b] = ((yc[a] >= 0) && (xc[b] >= 0)) ? ((yc[a] << 10) | xc[b]) : -1;
}

/* Distinct cells of one 32-sample cache line: entries grouped by slot (slot order), within a slot
 * in order of the HIGHEST lane holding the cell.  The reference's cell_analysis marks a cell at the
 * lane where (match_any mask >> lane) == 1, i.e. at its highest lane (PointingPlan.cu:27-35), and the
 * ring buffer takes the marked lanes in lane order (__fns, :71-73).
 * Returns the entry count; na[k] gets per-slot counts. */
static int line_cells(const float *xp, int64_t nsamp, int64_t icl, int ny, int nx, int periodic,
                      int cells_out[192], int na[6], uint32_t *err)
{
    int slots[32][6];
    for (int lane = 0; lane < 32; lane++) {
        int64_t s = 32 * icl + lane;
        int iy0, iy1, ix0, ix1;
        float dy, dx;
        *err |= locate_f32(xp[s], xp[s + nsamp], ny, nx, periodic, &iy0, &iy1, &ix0, &ix1, &dy, &dx);
        sample_slots(iy0, iy1, ix0, ix1, slots[lane]);
    }
    int n = 0;
    for (int k = 0; k < 6; k++) {
        int n0 = n;
        for (int lane = 0; lane < 32; lane++) {
            int c = slots[lane][k];
            if (c < 0) continue;
            int later = 0;
            for (int j = lane + 1; j < 32; j++)
                if (slots[j][k] == c) { later = 1; break; }
            if (!later) cells_out[n++] = c;
        }
        na[k] = n - n0;
    }
    return n;
}

static void preplan_geometry(int64_t nsamp, int64_t *ncl_per_tb, int64_t *nblocks)
{
    /* PointingPrePlan.cu:162-165 */
    int64_t ncl = (nsamp + 31) / 32;
    int64_t c = (ncl + 1023) / 1024;
    c = (c > 16) ? c : 16;
    c = (c + 3) & ~3LL;
    *ncl_per_tb = c;
    *nblocks = (ncl + c - 1) / c;
}

static int nsamp_ok(int64_t nsamp) { return (nsamp > 0) && (nsamp <= (1LL << 31)) && (nsamp % 32 == 0); }

void oracle_sample_slots(const float *xp, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic, int32_t *slots_out)
{
    for (int64_t s = 0; s < nsamp; s++) {
        int iy0, iy1, ix0, ix1, sl[6];
        float dy, dx;
        locate_f32(xp[s], xp[s + nsamp], ny, nx, periodic, &iy0, &iy1, &ix0, &ix1, &dy, &dx);
        sample_slots(iy0, iy1, ix0, ix1, sl);
        for (int k = 0; k < 6; k++)
            slots_out[6 * s + k] = sl[k];
    }
}

void oracle_line_counts(const float *xp, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic, uint8_t *counts)
{
    int cells[192], na[6];
    uint32_t err = 0;
    for (int64_t l = 0; l < nsamp / 32; l++)
        counts[l] = (uint8_t) line_cells(xp, nsamp, l, ny, nx, periodic, cells, na, &err);
}

int64_t oracle_preplan(const float *xp, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                       uint32_t *nmt_cumsum, int64_t *geom, uint32_t *err_out)
{
    if (!nsamp_ok(nsamp)) return -1;
    int64_t nclpb, nblocks;
    preplan_geometry(nsamp, &nclpb, &nblocks);
    int64_t ncl = nsamp / 32, nmt = 0;
    uint32_t err = 0;
    int cells[192], na[6];
    for (int64_t b = 0; b < nblocks; b++) {
        int64_t l1 = (b + 1) * nclpb;
        l1 = (l1 < ncl) ? l1 : ncl;
        for (int64_t l = b * nclpb; l < l1; l++)
            nmt += line_cells(xp, nsamp, l, ny, nx, periodic, cells, na, &err);
        nmt_cumsum[b] = (uint32_t) nmt;
    }
    for (int64_t b = nblocks; b < 1024; b++)
        nmt_cumsum[b] = (uint32_t) nmt;
    /* PointingPrePlan.cu:236-238 */
    int64_t nmt_per_tb = (int64_t) sqrt((double) nmt);
    nmt_per_tb = (nmt_per_tb + 32) & ~31LL;
    geom[0] = nclpb;
    geom[1] = nblocks;
    geom[2] = nmt_per_tb;
    geom[3] = (nmt + nmt_per_tb - 1) / nmt_per_tb;
    *err_out = err;
    return nmt;
}

uint32_t oracle_plan(const float *xp, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic,
                     int64_t nmt, uint64_t *plan_mt, uint32_t *owner_bits)
{
    if (!nsamp_ok(nsamp)) return ORACLE_ERR_INCONSISTENT_NMT;
    int64_t nclpb, nblocks;
    preplan_geometry(nsamp, &nclpb, &nblocks);
    int64_t ncl = nsamp / 32;

    uint64_t *unsorted = (uint64_t *) malloc(sizeof(uint64_t) * (nmt > 0 ? nmt : 1));
    uint32_t *owner_cell = (uint32_t *) malloc(sizeof(uint32_t) * (ncl > 0 ? ncl : 1));
    int64_t n = 0;
    uint32_t err = 0;
    int cells[192], na[6];

    for (int64_t b = 0; b < nblocks; b++) {
        int64_t l0 = b * nclpb, l1 = (b + 1) * nclpb;
        l1 = (l1 < ncl) ? l1 : ncl;
        /* Warp w of the reference's plan_kernel (W=4) handles lines l0+w, l0+w+4, ...
         * (PointingPlan.cu:167); its ring-buffer fill 'nmt_local' persists across those lines. */
        int nmt_local[4] = {0, 0, 0, 0};
        for (int64_t l = l0; l < l1; l++) {
            int w = (int) ((l - l0) & 3);
            int cnt = line_cells(xp, nsamp, l, ny, nx, periodic, cells, na, &err);
            int mflag = (cnt > 1);
            int na_cumul = 0, pos = 0;
            uint32_t minc = 0xffffffffu;
            for (int k = 0; k < 6; k++) {
                if (na[k] == 0) continue;
                /* mt_ringbuf::absorb (PointingPlan.cu:60-117): the first entry of this slot gets
                 * zflag iff mflag and no flush has happened yet on this line. */
                int zflag = mflag && (na_cumul == 0);
                for (int j = 0; j < na[k]; j++) {
                    uint64_t c = (uint64_t) cells[pos + j];
                    uint64_t word = c | ((uint64_t) l << 20);
                    if (mflag) word |= (1ULL << 46);
                    if (zflag && (j == 0)) word |= (1ULL << 47);
                    if (n < nmt) unsorted[n] = word;
                    n++;
                    if ((uint32_t) c < minc) minc = (uint32_t) c;
                }
                pos += na[k];
                nmt_local[w] += na[k];
                if (nmt_local[w] >= 32) {
                    nmt_local[w] -= 32;
                    na_cumul += na[k];
                }
            }
            owner_cell[l] = minc;
        }
    }

    if (n != nmt) {
        free(unsorted);
        free(owner_cell);
        return err | ORACLE_ERR_INCONSISTENT_NMT;
    }

    /* Stable counting sort by cell (bits 0-19): canonical (cell, cache line) order. */
    int64_t *count = (int64_t *) calloc((1 << 20) + 1, sizeof(int64_t));
    for (int64_t i = 0; i < nmt; i++)
        count[(unsorted[i] & 0xfffff) + 1]++;
    for (int64_t c = 0; c < (1 << 20); c++)
        count[c + 1] += count[c];
    for (int64_t i = 0; i < nmt; i++)
        plan_mt[count[unsorted[i] & 0xfffff]++] = unsorted[i];

    int64_t nwords = (nmt + 31) / 32;
    memset(owner_bits, 0, sizeof(uint32_t) * nwords);
    for (int64_t i = 0; i < nmt; i++) {
        uint64_t cl = (plan_mt[i] >> 20) & ((1ULL << 26) - 1);
        if ((uint32_t) (plan_mt[i] & 0xfffff) == owner_cell[cl])
            owner_bits[i >> 5] |= (1u << (i & 31));
    }

    free(count);
    free(unsorted);
    free(owner_cell);
    return err;
}
