// Per-sample pixel quantization for the PointingPlanTester test utility (the reference's
// quantize_kernel, kmsmith137/gpu_mm src_lib/PointingPlanTester.cu:22-63): the (iy0, ix0) of each
// sample's bilinear footprint, computed with the same locate() as every other kernel here so that
// roundoff agrees with the plan and the operators.
#include <algorithm>

#include "gmm_internal.hpp"

namespace gmm {
namespace {

__global__ void __launch_bounds__(256)
quantize_kernel(const float *__restrict__ xp, int64_t nsamp, int ny, int nx, bool periodic, int32_t *__restrict__ iypix,
                int32_t *__restrict__ ixpix, uint32_t *__restrict__ errword)
{
    __shared__ uint32_t s_err[8];
    uint32_t err = 0;
    for (int64_t s = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; s < nsamp; s += (int64_t) gridDim.x * blockDim.x) {
        Located L;
        err |= locate(__ldg(xp + s), __ldg(xp + nsamp + s), ny, nx, periodic, L);
        iypix[s] = L.iy0;
        ixpix[s] = L.ix0;
    }
    block_publish_err(err, s_err, errword);
}

}  // namespace
}  // namespace gmm

using namespace gmm;

extern "C" int gmm_quantize_pointing(const float *xpointing, int64_t nsamp, int32_t nypix_global, int32_t nxpix_global,
                                     int32_t periodic_xcoord, int32_t *iypix, int32_t *ixpix, uint32_t *errword,
                                     cudaStream_t stream)
{
    if (!xpointing || !iypix || !ixpix || !errword || (nsamp <= 0) || (nypix_global < 2) || (nxpix_global < 2))
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "quantize_pointing: bad argument");
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess) {
        const int64_t g = std::max<int64_t>(1, std::min<int64_t>((nsamp + 255) / 256, 8 * (int64_t) device_sm_count()));
        quantize_kernel<<<(unsigned) g, 256, 0, stream>>>(xpointing, nsamp, nypix_global, nxpix_global,
                                                          periodic_xcoord != 0, iypix, ixpix, errword);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess)
        return gmm_fail_message(GMM_ERR_CUDA, (std::string("quantize_pointing: ") + cudaGetErrorString(e)).c_str());
    return 0;
}
