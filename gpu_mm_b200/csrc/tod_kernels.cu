// TOD preprocessing on the device: deglitching (border means, jump removal), cut ranges
// (extract / insert / clear) and in-place clipping.
//
// Semantics follow the reference (kmsmith137/gpu_mm src_lib/deglitching.cu:61-210, cuts.cu:16-55,
// misc.cu:8-19, and the Python reference implementations gpu_mm.py:1507-1568).  Unlike the
// reference's kernels, every index read from an index map is checked against the arrays' extents:
// an entry out of range is skipped and sets bit 1 of the error word, so a bad map cannot write
// outside the arrays.
#include <algorithm>
#include <string>

#include "gmm_internal.hpp"

namespace gmm {
namespace {

constexpr uint32_t kErrRange = 1u;

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(kFullMask, v, o);
    return v;
}

// One warp per range r: the means of signal[di, b00:b01] and signal[di, b10:b11]; an empty range
// takes the other range's mean (deglitching.cu:61-96).
__global__ void __launch_bounds__(256)
border_means_kernel(float *__restrict__ out, const float *__restrict__ signal, int64_t ndet, int64_t nt,
                    const int32_t *__restrict__ index_map, int64_t R, uint32_t *__restrict__ errword)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t) gridDim.x * (blockDim.x >> 5);
    for (int64_t r = blockIdx.x * (int64_t) (blockDim.x >> 5) + (threadIdx.x >> 5); r < R; r += nwarps) {
        const int64_t di = index_map[5 * r], b00 = index_map[5 * r + 1], b01 = index_map[5 * r + 2];
        const int64_t b10 = index_map[5 * r + 3], b11 = index_map[5 * r + 4];
        const bool ok = (di >= 0) && (di < ndet) && (b00 >= 0) && (b01 <= nt) && (b10 >= 0) && (b11 <= nt);
        if (!ok) {
            if (lane == 0)
                atomicOr(errword, kErrRange);
            continue;
        }
        const float *s = signal + di * nt;
        float s0 = 0.0f, s1 = 0.0f;
        for (int64_t t = b00 + lane; t < b01; t += 32)
            s0 += s[t];
        for (int64_t t = b10 + lane; t < b11; t += 32)
            s1 += s[t];
        s0 = warp_sum(s0);
        s1 = warp_sum(s1);
        if (b00 < b01)
            s0 /= (float) (b01 - b00);
        if (b10 < b11)
            s1 /= (float) (b11 - b10);
        if (b00 >= b01)
            s0 = s1;
        if (b10 >= b11)
            s1 = s0;
        if (lane == 0) {
            out[2 * r] = s0;
            out[2 * r + 1] = s1;
        }
    }
}

// cumj = inclusive prefix sum of bvals[:,1] - bvals[:,0] (float, in order), by one CTA.
__global__ void __launch_bounds__(1024)
jump_cumsum_kernel(float *__restrict__ cumj, const float *__restrict__ bvals, int64_t R)
{
    __shared__ float s_part[32];
    __shared__ float s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        s_carry = 0.0f;
    __syncthreads();
    for (int64_t base = 0; base < R; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        float v = (i < R) ? (bvals[2 * i + 1] - bvals[2 * i]) : 0.0f;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float u = __shfl_up_sync(kFullMask, v, o);
            if (lane >= o)
                v += u;
        }
        if (lane == 31)
            s_part[warp] = v;
        __syncthreads();
        if (warp == 0) {
            float w = (lane < (int) (blockDim.x >> 5)) ? s_part[lane] : 0.0f;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float u = __shfl_up_sync(kFullMask, w, o);
                if (lane >= o)
                    w += u;
            }
            s_part[lane] = w;
        }
        __syncthreads();
        const float off = s_carry + ((warp > 0) ? s_part[warp - 1] : 0.0f);
        if (i < R)
            cumj[i] = off + v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1)
            s_carry = off + v;
        __syncthreads();
    }
}

// One CTA per range r (deglitching.cu:143-178): with dc = cumj[r] - cumj[r0-1],
// signal[di, t1:t2] = bvals[r,1] - dc and signal[di, t2:t3] -= dc, where t3 is the next range's start
// if it has the same detector, else nt.
__global__ void __launch_bounds__(128)
deglitch_kernel(float *__restrict__ signal, int64_t ndet, int64_t nt, const float *__restrict__ bvals,
                const float *__restrict__ cumj, const int32_t *__restrict__ index_map2, int64_t R,
                uint32_t *__restrict__ errword)
{
    for (int64_t r = blockIdx.x; r < R; r += gridDim.x) {
        const int64_t di = index_map2[4 * r], r0 = index_map2[4 * r + 1];
        const int64_t t1 = index_map2[4 * r + 2], t2 = index_map2[4 * r + 3];
        int64_t t3 = nt;
        if ((r < R - 1) && (index_map2[4 * r + 4] == di))
            t3 = index_map2[4 * r + 6];
        const bool ok = (di >= 0) && (di < ndet) && (r0 >= 0) && (r0 <= r) && (t1 >= 0) && (t1 <= t2) && (t2 <= nt) &&
                        (t3 <= nt);
        if (!ok) {
            if (threadIdx.x == 0)
                atomicOr(errword, kErrRange);
            continue;
        }
        const float dc = cumj[r] - ((r0 > 0) ? cumj[r0 - 1] : 0.0f);
        const float fill = bvals[2 * r + 1] - dc;
        float *s = signal + di * nt;
        for (int64_t t = t1 + threadIdx.x; t < t2; t += blockDim.x)
            s[t] = fill;
        for (int64_t t = t2 + threadIdx.x; t < t3; t += blockDim.x)
            s[t] -= dc;
    }
}

// Cut ranges (cuts.cu:16-36): range r is tod[det[r], istart[r] : istart[r]+len[r]], stored in rdata
// at ostart[r].  mode 0 extract (rdata <- tod), 1 insert (tod <- rdata), 2 clear (tod <- 0).
__global__ void __launch_bounds__(128)
ranges_kernel(int mode, float *__restrict__ tod, int64_t ndet, int64_t nsamp, float *__restrict__ rdata,
              int64_t nrdata, const int32_t *__restrict__ ostart, const int32_t *__restrict__ det,
              const int32_t *__restrict__ istart, const int32_t *__restrict__ len, int64_t nrange,
              uint32_t *__restrict__ errword)
{
    for (int64_t r = blockIdx.x; r < nrange; r += gridDim.x) {
        const int64_t d = det[r], i0 = istart[r], n = len[r];
        const int64_t o = (mode == 2) ? 0 : ostart[r];
        const bool ok = (d >= 0) && (d < ndet) && (i0 >= 0) && (n >= 0) && (i0 + n <= nsamp) &&
                        ((mode == 2) || ((o >= 0) && (o + n <= nrdata)));
        if (!ok) {
            if (threadIdx.x == 0)
                atomicOr(errword, kErrRange);
            continue;
        }
        float *t = tod + d * nsamp + i0;
        for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
            if (mode == 0)
                rdata[o + i] = t[i];
            else if (mode == 1)
                t[i] = rdata[o + i];
            else
                t[i] = 0.0f;
        }
    }
}

// arr = max(vmin, min(vmax, arr)) in place (misc.cu:8-19).
__global__ void __launch_bounds__(256)
clip_kernel(float *__restrict__ arr, int64_t n, float vmin, float vmax)
{
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        arr[i] = fmaxf(vmin, fminf(vmax, arr[i]));
}

int grid_for(int64_t work)
{
    return (int) std::max<int64_t>(1, std::min<int64_t>(work, 16 * (int64_t) device_sm_count()));
}

int finish(cudaError_t e, const char *where)
{
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string(where) + ": " + cudaGetErrorString(e)).c_str());
    return 0;
}

}  // namespace
}  // namespace gmm

using namespace gmm;

extern "C" {

int gmm_get_border_means(float *out, const float *signal, int64_t ndet, int64_t nt, const int32_t *index_map,
                         int64_t R, uint32_t *errword, cudaStream_t stream)
{
    if (!out || !signal || !index_map || !errword || (ndet < 0) || (nt < 0) || (R < 0))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "get_border_means: bad argument");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if ((e == cudaSuccess) && (R > 0))
        border_means_kernel<<<grid_for((R + 7) / 8), 256, 0, stream>>>(out, signal, ndet, nt, index_map, R, errword);
    return finish(e, "get_border_means");
}

int gmm_deglitch(float *signal, int64_t ndet, int64_t nt, const float *bvals, const int32_t *index_map2, int64_t R,
                 float *cumj, uint32_t *errword, cudaStream_t stream)
{
    if (!signal || !bvals || !index_map2 || !cumj || !errword || (ndet < 0) || (nt < 0) || (R < 0))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "deglitch: bad argument");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if ((e == cudaSuccess) && (R > 0)) {
        jump_cumsum_kernel<<<1, 1024, 0, stream>>>(cumj, bvals, R);
        deglitch_kernel<<<grid_for(R), 128, 0, stream>>>(signal, ndet, nt, bvals, cumj, index_map2, R, errword);
    }
    return finish(e, "deglitch");
}

int gmm_deglitch_cumj(float *signal, int64_t ndet, int64_t nt, const float *bvals, const float *cumj,
                      const int32_t *index_map2, int64_t R, uint32_t *errword, cudaStream_t stream)
{
    if (!signal || !bvals || !index_map2 || !cumj || !errword || (ndet < 0) || (nt < 0) || (R < 0))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "deglitch: bad argument");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if ((e == cudaSuccess) && (R > 0))
        deglitch_kernel<<<grid_for(R), 128, 0, stream>>>(signal, ndet, nt, bvals, cumj, index_map2, R, errword);
    return finish(e, "deglitch");
}

static int ranges(int mode, float *tod, int64_t ndet, int64_t nsamp, float *rdata, int64_t nrdata,
                  const int32_t *ostart, const int32_t *det, const int32_t *istart, const int32_t *len, int64_t nrange,
                  uint32_t *errword, cudaStream_t stream, const char *where)
{
    if (!tod || !det || !istart || !len || !errword || (mode != 2 && (!rdata || !ostart)) || (ndet < 0) ||
        (nsamp < 0) || (nrange < 0))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, (std::string(where) + ": bad argument").c_str());
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if ((e == cudaSuccess) && (nrange > 0))
        ranges_kernel<<<grid_for(nrange), 128, 0, stream>>>(mode, tod, ndet, nsamp, rdata, nrdata, ostart, det,
                                                            istart, len, nrange, errword);
    return finish(e, where);
}

int gmm_extract_ranges(const float *tod, int64_t ndet, int64_t nsamp, float *rdata, int64_t nrdata,
                       const int32_t *ostart, const int32_t *det, const int32_t *istart, const int32_t *len,
                       int64_t nrange, uint32_t *errword, cudaStream_t stream)
{
    return ranges(0, (float *) tod, ndet, nsamp, rdata, nrdata, ostart, det, istart, len, nrange, errword, stream,
                  "extract_ranges");
}

int gmm_insert_ranges(float *tod, int64_t ndet, int64_t nsamp, const float *rdata, int64_t nrdata,
                      const int32_t *ostart, const int32_t *det, const int32_t *istart, const int32_t *len,
                      int64_t nrange, uint32_t *errword, cudaStream_t stream)
{
    return ranges(1, tod, ndet, nsamp, (float *) rdata, nrdata, ostart, det, istart, len, nrange, errword, stream,
                  "insert_ranges");
}

int gmm_clear_ranges(float *tod, int64_t ndet, int64_t nsamp, const int32_t *det, const int32_t *istart,
                     const int32_t *len, int64_t nrange, uint32_t *errword, cudaStream_t stream)
{
    return ranges(2, tod, ndet, nsamp, nullptr, 0, nullptr, det, istart, len, nrange, errword, stream, "clear_ranges");
}

int gmm_clip(float *arr, int64_t n, float vmin, float vmax, cudaStream_t stream)
{
    if (!arr || (n < 0))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "clip: bad argument");
    if (n > 0)
        clip_kernel<<<grid_for((n + 255) / 256), 256, 0, stream>>>(arr, n, vmin, vmax);
    return finish(cudaSuccess, "clip");
}

}  // extern "C"
