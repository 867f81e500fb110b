// Plan construction without caller-provided temporary memory (gmm_plan_build_noalloc).
//
// The temporary storage of gmm_plan_build lives in a static __device__ array of this file.  Host
// code may not pass the array's name to a kernel (on the host it is only a stand-in symbol), so its
// device address is looked up once per device with cudaGetSymbolAddress and cached.
#include <mutex>
#include <sstream>
#include <string>

#include "gmm_internal.hpp"

namespace {

constexpr size_t kScratchBytes = (size_t) GMM_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_plan_scratch[kScratchBytes];

constexpr int kMaxDevices = 128;
void *g_scratch_ptr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

}  // namespace

extern "C" int gmm_plan_build_noalloc(const gmm_preplan_info *info, const uint32_t *nmt_cumsum, const float *xp,
                                      void *buf, int64_t buf_nbytes, int32_t debug, cudaStream_t stream)
{
    if (!info)
        return gmm_fail_message(GMM_ERR_INVALID_ARGUMENT, "gmm_plan_build_noalloc: null preplan");
    if (info->plan_constructor_tmp_nbytes > (int64_t) kScratchBytes) {
        std::ostringstream ss;
        ss << "gmm_plan_build_noalloc: this plan needs " << info->plan_constructor_tmp_nbytes
           << " bytes of temporary storage, more than the " << kScratchBytes
           << "-byte static scratch; use gmm_plan_build with a caller-allocated tmp buffer";
        return gmm_fail_message(GMM_ERR_BUFFER_TOO_SMALL, ss.str().c_str());
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return gmm_fail_message(GMM_ERR_CUDA, "gmm_plan_build_noalloc: cudaGetDevice failed");
    void *ptr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_ptr[dev]) {
            e = cudaGetSymbolAddress(&ptr, g_plan_scratch);
            if (e != cudaSuccess) {
                std::string msg = std::string("gmm_plan_build_noalloc: cudaGetSymbolAddress failed: ") +
                                  cudaGetErrorString(e);
                return gmm_fail_message(GMM_ERR_CUDA, msg.c_str());
            }
            g_scratch_ptr[dev] = ptr;
        }
        ptr = g_scratch_ptr[dev];
    }
    return gmm_plan_build(info, nmt_cumsum, xp, buf, buf_nbytes, ptr, (int64_t) kScratchBytes, debug, stream);
}
