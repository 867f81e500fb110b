// Minimal stand-in for the part of kmsmith137/ksgpu that the reference's pointing-operator sources
// use (TEST INFRASTRUCTURE ONLY: it lets oracle/Makefile compile those sources, unchanged, into the
// comparator library oracle/_ref/libgpu_mm_refgpu.so).  ksgpu itself is neither vendored nor
// installed; this file is written from the call sites in the reference's src_lib/*.cu and
// include/gpu_mm.hpp, not from ksgpu's source.
//
// Array<T>: a strided n-d view with shared ownership of its memory and a location flag word.
#pragma once

#include <sys/types.h>   // uint, ulong (used throughout the reference)

#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace ksgpu {

// Location / initialisation flags.
enum {
    af_gpu = 0x1,        // device memory
    af_uhost = 0x2,      // pageable host memory
    af_rhost = 0x4,      // pinned host memory
    af_unified = 0x8,    // managed memory
    af_zero = 0x10,      // zero-initialise on allocation
};

inline bool af_on_gpu(int aflags) { return (aflags & (af_gpu | af_unified)) != 0; }
inline bool af_on_host(int aflags) { return (aflags & (af_uhost | af_rhost | af_unified)) != 0; }

constexpr int ArrayMaxDim = 8;

template<typename T>
struct Array {
    T *data = nullptr;
    int ndim = 0;
    long shape[ArrayMaxDim] = {0};
    long size = 0;
    long strides[ArrayMaxDim] = {0};   // in elements
    std::shared_ptr<void> base;
    int aflags = 0;

    Array() = default;

    Array(std::initializer_list<long> shp, int flags) { _allocate(std::vector<long>(shp), flags); }
    Array(const std::vector<long> &shp, int flags) { _allocate(shp, flags); }

    // Non-owning contiguous view of existing memory (used by the comparator's C driver).
    static Array<T> view(T *p, const std::vector<long> &shp, int flags)
    {
        Array<T> a;
        a._set_shape(shp);
        a.data = p;
        a.aflags = flags;
        return a;
    }

    bool shape_equals(std::initializer_list<long> shp) const
    {
        if ((long) shp.size() != ndim)
            return false;
        int d = 0;
        for (long n : shp)
            if (shape[d++] != n)
                return false;
        return true;
    }

    bool on_gpu() const { return af_on_gpu(aflags); }
    bool on_host() const { return af_on_host(aflags); }

    bool is_fully_contiguous() const
    {
        long expected = 1;
        for (int d = ndim - 1; d >= 0; d--) {
            if ((shape[d] != 1) && (strides[d] != expected))
                return false;
            expected *= shape[d];
        }
        return true;
    }

    std::string shape_str() const
    {
        std::stringstream ss;
        ss << "(";
        for (int d = 0; d < ndim; d++)
            ss << (d ? "," : "") << shape[d];
        ss << ((ndim == 1) ? ",)" : ")");
        return ss.str();
    }

    Array<T> to_gpu() const { return _copy_to(af_gpu); }
    Array<T> to_host() const { return _copy_to(af_rhost); }

    // Copies the contents of 'src' (same shape, both contiguous) into this array.
    void fill(const Array<T> &src) const
    {
        if ((src.size != size) || !is_fully_contiguous() || !src.is_fully_contiguous())
            throw std::runtime_error("ksgpu shim: Array::fill() needs contiguous arrays of equal size");
        if (cudaMemcpy(data, src.data, size * sizeof(T), cudaMemcpyDefault) != cudaSuccess)
            throw std::runtime_error("ksgpu shim: Array::fill(): cudaMemcpy failed");
    }

    void _set_shape(const std::vector<long> &shp)
    {
        if (shp.size() > (size_t) ArrayMaxDim)
            throw std::runtime_error("ksgpu shim: too many dimensions");
        ndim = (int) shp.size();
        size = 1;
        for (int d = ndim - 1; d >= 0; d--) {
            shape[d] = shp[d];
            strides[d] = size;
            size *= shp[d];
        }
    }

    void _allocate(const std::vector<long> &shp, int flags)
    {
        _set_shape(shp);
        aflags = flags;
        const size_t nbytes = std::max<size_t>(size * sizeof(T), 1);
        void *p = nullptr;
        if (flags & af_gpu) {
            if (cudaMalloc(&p, nbytes) != cudaSuccess)
                throw std::runtime_error("ksgpu shim: cudaMalloc failed");
            if ((flags & af_zero) && (cudaMemset(p, 0, nbytes) != cudaSuccess))
                throw std::runtime_error("ksgpu shim: cudaMemset failed");
            base = std::shared_ptr<void>(p, [](void *q) { cudaFree(q); });
        } else if (flags & af_unified) {
            if (cudaMallocManaged(&p, nbytes) != cudaSuccess)
                throw std::runtime_error("ksgpu shim: cudaMallocManaged failed");
            if (flags & af_zero)
                std::memset(p, 0, nbytes);
            base = std::shared_ptr<void>(p, [](void *q) { cudaFree(q); });
        } else if (flags & af_rhost) {
            if (cudaMallocHost(&p, nbytes) != cudaSuccess)
                throw std::runtime_error("ksgpu shim: cudaMallocHost failed");
            if (flags & af_zero)
                std::memset(p, 0, nbytes);
            base = std::shared_ptr<void>(p, [](void *q) { cudaFreeHost(q); });
        } else {
            p = std::calloc(nbytes, 1);
            if (!p)
                throw std::runtime_error("ksgpu shim: calloc failed");
            base = std::shared_ptr<void>(p, [](void *q) { std::free(q); });
        }
        data = (T *) p;
    }

    Array<T> _copy_to(int flags) const
    {
        if (!is_fully_contiguous())
            throw std::runtime_error("ksgpu shim: copies need a contiguous array");
        Array<T> a(std::vector<long>(shape, shape + ndim), flags);
        if (cudaMemcpy(a.data, data, size * sizeof(T), cudaMemcpyDefault) != cudaSuccess)
            throw std::runtime_error("ksgpu shim: cudaMemcpy failed");
        return a;
    }
};

}  // namespace ksgpu
