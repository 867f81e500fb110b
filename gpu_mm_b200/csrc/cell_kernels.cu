// Cell-level map transforms on the device: local map -> global map, and the cell broadcast / reduce
// of cell-major buffers used for map exchange.
//
// Semantics follow the reference's host functions (kmsmith137/gpu_mm src_lib/local_map_to_global.cu:12-44,
// cell_broadcast.cu:17-36, cell_reduce.cu:17-41); here they run as kernels on device arrays.
#include <algorithm>
#include <sstream>

#include "gmm_internal.hpp"

namespace gmm {
namespace {

constexpr int kCellFloats = 3 * 64 * 64;

// One CTA per (cell, plane): copies the cell's 64 x 64 block (clipped to the global map) from the
// local map into the dense (3, ny, nx) global map.  Pixels of absent cells are written by the
// zero-fill of the caller.
__global__ void __launch_bounds__(256)
local_to_global_kernel(float *__restrict__ dst, const float *__restrict__ src, const int64_t *__restrict__ cell_offsets,
                       int ny, int nx, int nycells, int nxcells, int64_t ystride, int64_t polstride)
{
    const int64_t ncell = (int64_t) nycells * nxcells;
    for (int64_t b = blockIdx.x; b < 3 * ncell; b += gridDim.x) {
        const int p = (int) (b / ncell);
        const int64_t c = b % ncell;
        const int64_t off = __ldg(cell_offsets + c);
        if (off < 0)
            continue;
        const int iy0 = (int) (c / nxcells) * 64, ix0 = (int) (c % nxcells) * 64;
        const int h = min(ny, iy0 + 64) - iy0, w = min(nx, ix0 + 64) - ix0;
        for (int k = threadIdx.x; k < h * 64; k += blockDim.x) {
            const int iy = k >> 6, ix = k & 63;
            if (ix < w)
                dst[(int64_t) p * ny * nx + (int64_t) (iy0 + iy) * nx + ix0 + ix] =
                    __ldg(src + off + p * polstride + iy * ystride + ix);
        }
    }
}

// dst cell i <- src cell index_map[i] (cell_broadcast); indices outside [0, nsrc_cells) are skipped
// and flagged.
__global__ void __launch_bounds__(256)
cell_broadcast_kernel(float *__restrict__ dst, const float *__restrict__ src, int64_t nsrc_cells,
                      const int64_t *__restrict__ index_map, int64_t ncells, uint32_t *__restrict__ errword)
{
    for (int64_t i = blockIdx.x; i < ncells; i += gridDim.x) {
        const int64_t j = __ldg(index_map + i);
        if ((j < 0) || (j >= nsrc_cells)) {
            if (threadIdx.x == 0)
                atomicOr(errword, 1u);
            continue;
        }
        const float4 *s = reinterpret_cast<const float4 *>(src + j * kCellFloats);
        float4 *d = reinterpret_cast<float4 *>(dst + i * kCellFloats);
        for (int k = threadIdx.x; k < kCellFloats / 4; k += blockDim.x)
            d[k] = __ldg(s + k);
    }
}

// dst cell index_map[i] += src cell i (cell_reduce; dst is zeroed by the caller, repeated indices
// accumulate); indices outside [0, ndst_cells) are skipped and flagged.
__global__ void __launch_bounds__(256)
cell_reduce_kernel(float *__restrict__ dst, int64_t ndst_cells, const float *__restrict__ src,
                   const int64_t *__restrict__ index_map, int64_t ncells, uint32_t *__restrict__ errword)
{
    for (int64_t i = blockIdx.x; i < ncells; i += gridDim.x) {
        const int64_t j = __ldg(index_map + i);
        if ((j < 0) || (j >= ndst_cells)) {
            if (threadIdx.x == 0)
                atomicOr(errword, 1u);
            continue;
        }
        const float *s = src + i * kCellFloats;
        float *d = dst + j * kCellFloats;
        for (int k = threadIdx.x; k < kCellFloats; k += blockDim.x)
            atomicAdd(d + k, __ldg(s + k));
    }
}

int grid_for(int64_t work)
{
    return (int) std::max<int64_t>(1, std::min<int64_t>(work, 16 * (int64_t) device_sm_count()));
}

}  // namespace
}  // namespace gmm

using namespace gmm;

extern "C" {

int gmm_local_map_to_global(float *dst, const float *src, const gmm_lpix *lp, cudaStream_t stream)
{
    if (!dst || !src || !lp || !lp->cell_offsets)
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "local_map_to_global: null argument");
    const int64_t n = 3ll * lp->nypix_global * lp->nxpix_global;
    cudaError_t e = cudaMemsetAsync(dst, 0, n * sizeof(float), stream);
    if (e == cudaSuccess) {
        local_to_global_kernel<<<grid_for(3ll * lp->nycells * lp->nxcells), 256, 0, stream>>>(
            dst, src, lp->cell_offsets, lp->nypix_global, lp->nxpix_global, lp->nycells, lp->nxcells, lp->ystride,
            lp->polstride);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string("local_map_to_global: ") + cudaGetErrorString(e)).c_str());
    return 0;
}

int gmm_cell_broadcast(float *dst, const float *src, int64_t nsrc, const int64_t *index_map, int64_t ncells,
                       uint32_t *errword, cudaStream_t stream)
{
    if (!dst || !src || !index_map || !errword || (ncells < 0) || (nsrc < 0) || (nsrc % (3 * 64 * 64)) ||
        ((((uintptr_t) dst) | ((uintptr_t) src)) & 15))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT,
                                "cell_broadcast: need device arrays (16-byte aligned), nsrc a multiple of 3*64*64");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if ((e == cudaSuccess) && (ncells > 0)) {
        cell_broadcast_kernel<<<grid_for(ncells), 256, 0, stream>>>(dst, src, nsrc / (3 * 64 * 64), index_map, ncells,
                                                                    errword);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string("cell_broadcast: ") + cudaGetErrorString(e)).c_str());
    return 0;
}

int gmm_cell_reduce(float *dst, int64_t ndst, const float *src, const int64_t *index_map, int64_t ncells,
                    uint32_t *errword, cudaStream_t stream)
{
    if (!dst || !src || !index_map || !errword || (ncells < 0) || (ndst < 0) || (ndst % (3 * 64 * 64)))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "cell_reduce: need device arrays, ndst a multiple of 3*64*64");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(dst, 0, ndst * sizeof(float), stream);
    if ((e == cudaSuccess) && (ncells > 0)) {
        cell_reduce_kernel<<<grid_for(ncells), 256, 0, stream>>>(dst, ndst / (3 * 64 * 64), src, index_map, ncells,
                                                                 errword);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string("cell_reduce: ") + cudaGetErrorString(e)).c_str());
    return 0;
}

}  // extern "C"
