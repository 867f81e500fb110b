// Double-precision unplanned operators: the reference's launch_unplanned_map2tod<double> and
// launch_unplanned_tod2map<double> (kmsmith137/gpu_mm src_lib/map2tod_unplanned.cu:17-127,
// tod2map_unplanned.cu:17-121), whose arithmetic is pixel_locator<double>::locate,
// map_evaluator<double>::eval and map_accumulator<double>::accum (gpu_mm_internals.hpp:124-355).
// One sample per thread, grid-stride; map reads and float64 atomics go straight to global memory.
// The planned operators have no double form: the reference instantiates them, but their 96 KB
// of dynamic shared memory cannot be launched without an opt-in the reference does not make.
#include <algorithm>

#include "gmm_internal.hpp"

namespace gmm {
namespace {

struct F64Args {
    double *out;               // tod (map2tod) or local map (tod2map)
    const double *in;          // local map (map2tod) or tod (tod2map)
    const double *xp;          // xpointing [3][nsamp]
    const int64_t *cell_offsets;
    int64_t nsamp;
    int ny, nx;
    bool periodic;
    int nycells, nxcells;
    int64_t ystride, polstride;
    bool partial, accum;
    uint32_t *errword;
};

struct LocatedD {
    int iy0, iy1, ix0, ix1;
    double dy, dx;
};

// pixel_locator<double>::locate (gpu_mm_internals.hpp:124-164), the same steps as the float locate().
__device__ __forceinline__ uint32_t locate_d(double ypix, double xpix, int ny, int nx, bool periodic, LocatedD &L)
{
    uint32_t err = 0;
    int y0 = __double2int_rz(ypix);
    y0 = max(y0, 0);
    y0 = min(y0, ny - 2);
    L.iy0 = y0;
    L.iy1 = y0 + 1;
    L.dy = ypix - double(y0);
    const bool yvalid = (ypix >= 0.0) && (ypix <= double(ny - 1));
    err |= yvalid ? 0u : kErrBadYpix;
    if (periodic) {
        const bool xvalid = (xpix >= double(-nx)) && (xpix <= double(2 * nx));
        err |= xvalid ? 0u : kErrBadXpix;
        xpix = (xpix >= 0.0) ? xpix : (xpix + double(nx));
        xpix = (xpix <= double(nx)) ? xpix : (xpix - double(nx));
        int x0 = __double2int_rz(xpix);
        x0 = max(x0, 0);
        L.dx = xpix - double(x0);
        x0 = (x0 < nx) ? x0 : 0;
        const int x1 = x0 + 1;
        L.ix0 = x0;
        L.ix1 = (x1 < nx) ? x1 : 0;
    } else {
        const bool xvalid = (xpix >= 0.0) && (xpix <= double(nx - 2));
        err |= xvalid ? 0u : kErrBadXpix;
        int x0 = __double2int_rz(xpix);
        x0 = max(x0, 0);
        x0 = min(x0, nx - 2);
        L.ix0 = x0;
        L.ix1 = x0 + 1;
        L.dx = xpix - double(x0);
    }
    return err;
}

// Local-map offset of global pixel (iy, ix), or -1 if its cell is absent (map_evaluator addressing).
__device__ __forceinline__ int64_t pixel_offset_d(const F64Args &a, int iy, int ix)
{
    const int iyc = iy >> 6, ixc = ix >> 6;
    if ((iy < 0) || (ix < 0) || (iyc >= a.nycells) || (ixc >= a.nxcells))
        return -1;
    const int64_t off = __ldg(a.cell_offsets + (int64_t) iyc * a.nxcells + ixc);
    return (off < 0) ? -1 : off + (int64_t) (iy & 63) * a.ystride + (ix & 63);
}

__device__ __forceinline__ double eval_d(const F64Args &a, int iy, int ix, double c, double s, uint32_t &err)
{
    const int64_t off = pixel_offset_d(a, iy, ix);
    const bool valid = off >= 0;
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
    if (!valid)
        return 0.0;
    return a.in[off] + c * a.in[off + a.polstride] + s * a.in[off + 2 * a.polstride];
}

__device__ __forceinline__ void accum_d(const F64Args &a, int iy, int ix, double t, double c, double s, double w,
                                        uint32_t &err)
{
    const int64_t off = pixel_offset_d(a, iy, ix);
    const bool valid = off >= 0;
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
    if (valid) {
        atomicAdd(a.out + off, w * t);
        atomicAdd(a.out + off + a.polstride, w * t * c);
        atomicAdd(a.out + off + 2 * a.polstride, w * t * s);
    }
}

template<bool TOD2MAP>
__global__ void __launch_bounds__(256) unplanned_f64_kernel(F64Args a)
{
    __shared__ uint32_t s_err[8];
    uint32_t err = 0;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; s < a.nsamp; s += stride) {
        LocatedD L;
        err |= locate_d(a.xp[s], a.xp[a.nsamp + s], a.ny, a.nx, a.periodic, L);
        double sn, cs;
        sincos(2.0 * a.xp[2 * a.nsamp + s], &sn, &cs);
        const double w00 = (1.0 - L.dy) * (1.0 - L.dx), w01 = (1.0 - L.dy) * L.dx;
        const double w10 = L.dy * (1.0 - L.dx), w11 = L.dy * L.dx;
        if constexpr (TOD2MAP) {
            const double t = a.in[s];
            accum_d(a, L.iy0, L.ix0, t, cs, sn, w00, err);
            accum_d(a, L.iy0, L.ix1, t, cs, sn, w01, err);
            accum_d(a, L.iy1, L.ix0, t, cs, sn, w10, err);
            accum_d(a, L.iy1, L.ix1, t, cs, sn, w11, err);
        } else {
            double r = w00 * eval_d(a, L.iy0, L.ix0, cs, sn, err);
            r += w01 * eval_d(a, L.iy0, L.ix1, cs, sn, err);
            r += w10 * eval_d(a, L.iy1, L.ix0, cs, sn, err);
            r += w11 * eval_d(a, L.iy1, L.ix1, cs, sn, err);
            a.out[s] = a.accum ? (a.out[s] + r) : r;
        }
    }
    block_publish_err(err, s_err, a.errword);
}

int unplanned_f64(bool tod2map, double *out, const double *in, const double *xp, int64_t nsamp, const gmm_lpix *lp,
                  uint32_t *errflags, int64_t errflags_len, int32_t partial, int32_t accum, int32_t sync_check,
                  cudaStream_t stream, const char *where)
{
    if (!out || !in || !xp || !errflags || !lp || !lp->cell_offsets || (errflags_len < 1) || (nsamp <= 0) ||
        (lp->nypix_global < 2) || (lp->nxpix_global < 2))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT,
                                (std::string(where) + ": bad argument (null pointer, nsamp <= 0 or errflags_len < 1)").c_str());
    F64Args a;
    a.out = out;
    a.in = in;
    a.xp = xp;
    a.cell_offsets = lp->cell_offsets;
    a.nsamp = nsamp;
    a.ny = lp->nypix_global;
    a.nx = lp->nxpix_global;
    a.periodic = lp->periodic_xcoord != 0;
    a.nycells = lp->nycells;
    a.nxcells = lp->nxcells;
    a.ystride = lp->ystride;
    a.polstride = lp->polstride;
    a.partial = partial != 0;
    a.accum = accum != 0;
    a.errword = errflags;
    cudaError_t e = cudaMemsetAsync(errflags, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess) {
        const int64_t g = std::max<int64_t>(1, std::min<int64_t>((nsamp + 255) / 256, 8 * (int64_t) device_sm_count()));
        if (tod2map)
            unplanned_f64_kernel<true><<<(unsigned) g, 256, 0, stream>>>(a);
        else
            unplanned_f64_kernel<false><<<(unsigned) g, 256, 0, stream>>>(a);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string(where) + ": " + cudaGetErrorString(e)).c_str());
    if (!sync_check)
        return 0;
    uint32_t h = 0;
    e = cudaMemcpyAsync(&h, errflags, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string(where) + ": " + cudaGetErrorString(e)).c_str());
    return report_err_bits(h, where, partial ? GMM_ERR_NOT_IN_PIXELIZATION : 0u);
}

}  // namespace
}  // namespace gmm

using namespace gmm;

extern "C" {

int gmm_unplanned_map2tod_f64(double *tod, const double *local_map, const double *xpointing, int64_t nsamp,
                              const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                              int32_t partial_pixelization, int32_t accum, int32_t sync_check, cudaStream_t stream)
{
    return unplanned_f64(false, tod, local_map, xpointing, nsamp, lpix, errflags_gpu, errflags_len,
                         partial_pixelization, accum, sync_check, stream, "unplanned_map2tod");
}

int gmm_unplanned_tod2map_f64(double *local_map, const double *tod, const double *xpointing, int64_t nsamp,
                              const gmm_lpix *lpix, uint32_t *errflags_gpu, int64_t errflags_len,
                              int32_t partial_pixelization, int32_t sync_check, cudaStream_t stream)
{
    return unplanned_f64(true, local_map, tod, xpointing, nsamp, lpix, errflags_gpu, errflags_len,
                         partial_pixelization, 0, sync_check, stream, "unplanned_tod2map");
}

}  // extern "C"
