// Device building blocks shared by the gpu_mm_b200 kernels (sm_100a).
//
// The per-sample arithmetic restates the reference's pixel_locator / cell_enumerator
// (kmsmith137/gpu_mm include/gpu_mm_internals.hpp:104-237); the rest is this implementation's own.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gmm {

constexpr uint32_t kErrBadYpix = 0x1;
constexpr uint32_t kErrBadXpix = 0x2;
constexpr uint32_t kErrInconsistentNmt = 0x4;
constexpr uint32_t kErrNotInPixelization = 0x8;
constexpr unsigned kFullMask = 0xffffffffu;

// mt word layout (PointingPlan.cu:75-80): bits 0-9 ixcell, 10-19 iycell, 20-45 cache line,
// 46 mflag (line touches more than one cell), 47 zflag.
constexpr int kCellBits = 20;
constexpr uint64_t kCellMask = (1ull << 20) - 1;
constexpr uint64_t kClMask = (1ull << 26) - 1;
constexpr uint64_t kMflag = 1ull << 46;
constexpr uint64_t kZflag = 1ull << 47;

// Owner words of single-TOD plans (one per cache line: its lowest cell | line << 20 | mflag << 46)
// carry the line's row band in bits 48-53: the lowest row of its samples' upper bilinear neighbours
// (locate's row clamped to [0, ny - 2]), relative to the owner cell's first row, clamped to [0, 63].  The owner list is sorted by
// (cell, band, line).
constexpr int kBandShift = 48;
constexpr int kBandBits = 6;

struct Located {
    int iy0, iy1, ix0, ix1;
    float dy, dx;
};

// pixel_locator<float>::locate (gpu_mm_internals.hpp:124-164): global pixel coordinates of the
// four bilinear neighbours.  Bad coordinates set error bits but still give in-range indices.
__device__ __forceinline__ uint32_t locate(float ypix, float xpix, int ny, int nx, bool periodic, Located &L)
{
    uint32_t err = 0;
    int y0 = __float2int_rz(ypix);   // truncation; NaN gives 0
    y0 = max(y0, 0);
    y0 = min(y0, ny - 2);
    L.iy0 = y0;
    L.iy1 = y0 + 1;
    L.dy = ypix - float(y0);
    bool yvalid = (ypix >= 0.0f) && (ypix <= float(ny - 1));
    err |= yvalid ? 0u : kErrBadYpix;

    if (periodic) {
        bool xvalid = (xpix >= float(-nx)) && (xpix <= float(2 * nx));
        err |= xvalid ? 0u : kErrBadXpix;
        xpix = (xpix >= 0.0f) ? xpix : (xpix + float(nx));
        xpix = (xpix <= float(nx)) ? xpix : (xpix - float(nx));
        int x0 = __float2int_rz(xpix);
        x0 = max(x0, 0);
        L.dx = xpix - float(x0);
        x0 = (x0 < nx) ? x0 : 0;
        int x1 = x0 + 1;
        L.ix0 = x0;
        L.ix1 = (x1 < nx) ? x1 : 0;
    } else {
        bool xvalid = (xpix >= 0.0f) && (xpix <= float(nx - 2));
        err |= xvalid ? 0u : kErrBadXpix;
        int x0 = __float2int_rz(xpix);
        x0 = max(x0, 0);
        x0 = min(x0, nx - 2);
        L.ix0 = x0;
        L.ix1 = x0 + 1;
        L.dx = xpix - float(x0);
    }
    return err;
}

// The six cell "slots" of a sample, restating cell_enumerator::enumerate
// (gpu_mm_internals.hpp:194-236) as a function of cell value: y-slot = iycell parity; x-slot 0 =
// even non-zero ixcell, 1 = odd, 2 = ixcell 0.  Slot k = 3*yslot + xslot is in the order
// ca0..ca5 of PointingPlan.cu:173-178.  Empty slots hold -1; filled ones (iycell << 10) | ixcell.
__device__ __forceinline__ void cell_slots(const Located &L, int slots[6])
{
    int iyc0 = L.iy0 >> 6, iyc1 = L.iy1 >> 6;
    int ixc0 = L.ix0 >> 6, ixc1 = L.ix1 >> 6;
    bool ysame = (iyc0 == iyc1);
    bool xsame = (ixc0 == ixc1);
    int yc[2], xc[3];
    // y-cells are consecutive (iy1 = iy0+1), so the two have opposite parities.
    yc[0] = (iyc0 & 1) ? (ysame ? -1 : iyc1) : iyc0;
    yc[1] = (iyc0 & 1) ? iyc0 : (ysame ? -1 : iyc1);
    int xs0 = (ixc0 == 0) ? 2 : (ixc0 & 1);
    int xs1 = (ixc1 == 0) ? 2 : (ixc1 & 1);
#pragma unroll
    for (int b = 0; b < 3; b++)
        xc[b] = (xs0 == b) ? ixc0 : ((!xsame && (xs1 == b)) ? ixc1 : -1);
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 3; b++)
            slots[3 * a + b] = ((yc[a] >= 0) && (xc[b] >= 0)) ? ((yc[a] << 10) | xc[b]) : -1;
}

// Per-slot warp analysis of one 32-sample cache line (the role of cell_analysis,
// PointingPlan.cu:19-37): amask[k] has one bit per distinct valid cell of slot k, at the highest lane
// holding it -- the reference marks the lane where (match_any mask >> lane) == 1 -- so that a slot's
// cells come in the reference's ring-buffer order (marked lanes in lane order), which decides which
// of them carries zflag.
__device__ __forceinline__ void line_slot_masks(const int slots[6], unsigned amask[6])
{
    const unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        unsigned peers = __match_any_sync(kFullMask, (unsigned) slots[k]);
        bool highest = (peers >> lane) == 1u;
        amask[k] = __ballot_sync(kFullMask, highest && (slots[k] >= 0));
    }
}

// sin(th) and cos(th) for |th| <= 1024: th is reduced to [-pi, pi] by a two-term Cody-Waite split of
// 2*pi (W. J. Cody and W. Waite, "Software Manual for the Elementary Functions", 1980): head
// 6.28125 (exact in 8 bits, so j*head is exact for |j| < 2^16) plus the float tail 2*pi - 6.28125;
// then the hardware approximations __sinf/__cosf.  Absolute error about 6e-7 against CUDA's sincosf
// (the hardware approximations' own error dominates; the tail term adds at most 163 * 2^-34).
__device__ __forceinline__ void sincos_reduced(float th, float *s, float *c)
{
    // j = rint(th / 2pi), rounded by adding and subtracting 1.5 * 2^23 (round-to-nearest-even on the
    // FMA pipe; exact for |th / 2pi| < 2^22), the same value rintf gives.
    const float j = __fadd_rn(__fadd_rn(__fmul_rn(th, 0.15915494309189535f), 12582912.0f), -12582912.0f);
    float r = fmaf(j, -6.28125f, th);
    r = fmaf(j, -1.9353071795864769e-3f, r);
    __sincosf(r, s, c);
}

// floor(v) of a float v in [0, 2^23) as an int, and as an exact float in *fv, without a conversion
// instruction: v + 2^23 rounded toward zero is 2^23 + floor(v), whose low mantissa bits are floor(v).
// For v >= 0 this is the truncation __float2int_rz(v) that locate() uses, bit for bit.
__device__ __forceinline__ int floor_nonneg(float v, float *fv)
{
    const float b = __fadd_rz(v, 8388608.0f);
    *fv = __fadd_rn(b, -8388608.0f);
    return __float_as_int(b) - 0x4B000000;
}

// sin(2a) and cos(2a) for the detector response: sincos_reduced for |2a| <= 1024, sincosf beyond.
__device__ __forceinline__ void sincos2a(float alpha, float *s, float *c)
{
    const float th = 2.0f * alpha;
    if (fabsf(th) <= 1024.0f)
        sincos_reduced(th, s, c);
    else
        sincosf(th, s, c);
}

// Band word of a line of a single-TOD plan (one per owner entry, stored in owner-list order): the
// shape of the line as the tod2map band path needs it, computed once from the pointing when the
// plan is built.  The band path accumulates a line in the rows R0 .. R0 + 2 and the columns
// x0 + [0, 96) of its (cell, band) (R0 = 64 iycell + band, x0 = 64 ixcell); column k = floor(x) - x0.
//   bits 0-31  bit i set iff sample i lies in the same column as sample i - 1 (i >= 1)
//   bits 32-38 the first column in scan order, kmin (0..94)
//   bits 39-44 number of columns, ncol (1..32): the columns are kmin .. kmin + ncol - 1
//   bit  45    x increases along the line (scan order = lane order; else reversed)
//   bit  46    the line takes the band path (all conditions of band_line_word below hold)
//   bit  47    some column holds three or four consecutive samples
//   bit  48    the samples' upper rows are R0 and R0 + 1 (the line crosses a pixel row), not R0 only
constexpr int kBandKminShift = 32, kBandNcolShift = 39;
constexpr uint64_t kBandInc = 1ull << 45, kBandFast = 1ull << 46, kBandRun3 = 1ull << 47, kBandTwoRows = 1ull << 48;

// The band word of one cache line, by the full warp (lane = sample).  The line takes the band path
// (bit 46) iff every sample has y in [R0, R0 + 2) -- upper neighbours in row R0 or R0 + 1 -- with
// the rows inside the map (R0 <= ny - 2 if all are in R0, else R0 <= ny - 3: no clamp in locate),
// x in [x0, x0 + 95) and x < x_hi (nx if periodic: no fold; nx - 2 otherwise: in range), and the
// column moves along the line in one direction by 0 or 1 per sample, stays in one column for at
// most four consecutive samples (two if the line crosses a row), and repeats at least once (so the
// line spans at most 32 columns).  dy = y - R0 and xr = x - x0 are exact; non-negative floats
// compare as unsigned integers (negative values and NaN fail).  The word is 0 when the line does
// not take the path.
__device__ __forceinline__ uint64_t band_line_word(float y, float x, int R0, int x0, int ny, float x_hi)
{
    const int lane = threadIdx.x & 31;
    const float dy = y - (float) R0;
    const float xr = x - (float) x0;
    const bool two = __any_sync(kFullMask, (unsigned) __float_as_int(dy) >= 0x3f800000u);
    const bool ok = (R0 <= ny - (two ? 3 : 2)) && ((unsigned) __float_as_int(dy) < 0x40000000u) &&
                    ((unsigned) __float_as_int(xr) < 0x42be0000u) &&
                    ((unsigned) __float_as_int(x) < (unsigned) __float_as_int(x_hi));
    const int k = (int) floorf(xr);
    const int dk = k - __shfl_up_sync(kFullMask, k, 1);
    const unsigned su = __ballot_sync(kFullMask, (lane > 0) && (dk == 0));
    const unsigned up = __ballot_sync(kFullMask, (lane > 0) && (dk == 1));
    const unsigned down = __ballot_sync(kFullMask, (lane > 0) && (dk == -1));
    const unsigned bad = __ballot_sync(kFullMask, !ok);
    const unsigned r3 = su & (su >> 1);
    const int k0 = __shfl_sync(kFullMask, k, 0), k31 = __shfl_sync(kFullMask, k, 31);
    if ((bad != 0u) || ((su | up | down) != 0xfffffffeu) || ((up != 0u) && (down != 0u)) || (su == 0u) ||
        ((r3 & (r3 >> 2)) != 0u) || (two && (r3 != 0u)))
        return 0ull;
    const bool inc = down == 0u;
    const int kmin = inc ? k0 : k31;
    const int ncol = (inc ? k31 : k0) - kmin + 1;
    return (uint64_t) su | ((uint64_t) kmin << kBandKminShift) | ((uint64_t) ncol << kBandNcolShift) |
           (inc ? kBandInc : 0ull) | kBandFast | ((r3 != 0u) ? kBandRun3 : 0ull) | (two ? kBandTwoRows : 0ull);
}

// OR-reduce an error word over the block and publish it with one atomicOr per block (only if
// non-zero).  'scratch' needs blockDim.x/32 words; must be called by all threads of the block.
__device__ __forceinline__ void block_publish_err(uint32_t err, uint32_t *scratch, uint32_t *errword)
{
    err = __reduce_or_sync(kFullMask, err);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    if (lane == 0)
        scratch[warp] = err;
    __syncthreads();
    if (warp == 0) {
        uint32_t e = (lane < nwarps) ? scratch[lane] : 0u;
        e = __reduce_or_sync(kFullMask, e);
        if ((lane == 0) && (e != 0))
            atomicOr(errword, e);
    }
}

}  // namespace gmm
