// Minimal stand-in for ksgpu's CUDA error macros (TEST INFRASTRUCTURE ONLY; see Array.hpp).
#pragma once

#include <sstream>
#include <stdexcept>

#include <cuda_runtime.h>

#include "xassert.hpp"

#define CUDA_CALL(x) \
    do { \
        const cudaError_t e_ = (x); \
        if (e_ != cudaSuccess) { \
            std::stringstream ss_; \
            ss_ << "CUDA error: " << #x << ": " << cudaGetErrorString(e_) << " (" << __FILE__ << ":" << __LINE__ << ")"; \
            throw std::runtime_error(ss_.str()); \
        } \
    } while (0)

#define CUDA_PEEK(msg) \
    do { \
        const cudaError_t e_ = cudaPeekAtLastError(); \
        if (e_ != cudaSuccess) { \
            std::stringstream ss_; \
            ss_ << "CUDA error after " << (msg) << ": " << cudaGetErrorString(e_); \
            throw std::runtime_error(ss_.str()); \
        } \
    } while (0)
