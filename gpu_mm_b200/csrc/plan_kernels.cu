// Plan construction on sm_100a: preplan counts, deterministic mt emission, hand-written LSD
// radix sort, and dynamic-map cell discovery.
//
// Reference behaviour reproduced here (kmsmith137/gpu_mm):
//   PointingPrePlan.cu:17-108    per-block count of (cell, cache line) pairs -> nmt_cumsum
//   PointingPlan.cu:19-231       mt words, mflag and zflag (per-warp ring-buffer semantics)
//   PointingPlan.cu:300-309      stable sort of the mt words by cell (CUB there, hand-written here)
//   expand_dynamic_map.cu:18-102 cells of a sorted plan that are newly "targeted"
//
// Design: instead of the reference's racy chunk claims followed by a 20-bit sort (which leaves
// the within-cell order nondeterministic), the emit kernel writes every planner block's words in
// cache-line order, so the stable radix sort yields the canonical (cell, cache line) order and
// the plan is bit-reproducible.  zflag is derived in closed form from per-line counts: the
// reference's ring-buffer fill at the start of a line is the running count of that warp's
// earlier lines mod 32.
#include <algorithm>

#include "gmm_internal.hpp"

namespace gmm {

// ------------------------------------------------------------------------------------------------
// Preplan: per planner block, the number of distinct (cell, line) pairs.

constexpr int kPlanWarps = 8;          // warps per planner CTA
constexpr int kLinesPerWarp = 4;       // lines per warp per round
constexpr int kRoundLines = kPlanWarps * kLinesPerWarp;   // 32: one scan per round

static_assert(kRoundLines == 32, "round scan assumes one line per lane");

struct LineSlots {
    int slots[6];
    unsigned amask[6];
};

// Slot analysis of one cache line by the full warp; returns its number of (cell, line) pairs.
// A line whose samples all have their four bilinear neighbours in one and the same cell (most lines:
// a line is 32 samples, a cell 64 pixels wide) has exactly one pair, the same result the six-slot
// analysis gives it: that cell, reported in slot 0 at lane 0.  The test is two shifts and two
// compares per lane plus one shuffle and one vote, where the slot analysis is ALU-bound.
__device__ __forceinline__ int analyse_line(float y, float x, int ny, int nx, bool periodic, LineSlots &ls,
                                            uint32_t &err)
{
    Located L;
    err |= locate(y, x, ny, nx, periodic, L);
    const bool one = ((L.iy0 >> 6) == (L.iy1 >> 6)) && ((L.ix0 >> 6) == (L.ix1 >> 6));
    const int c = ((L.iy0 >> 6) << 10) | (L.ix0 >> 6);
    const int c0 = __shfl_sync(kFullMask, c, 0);
    if (__all_sync(kFullMask, one && (c == c0))) {
#pragma unroll
        for (int k = 0; k < 6; k++) {
            ls.slots[k] = (k == 0) ? c0 : -1;
            ls.amask[k] = (k == 0) ? 1u : 0u;
        }
        return 1;
    }
    cell_slots(L, ls.slots);
    line_slot_masks(ls.slots, ls.amask);
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < 6; k++)
        cnt += __popc(ls.amask[k]);
    return cnt;
}

// Number of (cell, line) pairs of one cache line for the preplan, by the full warp.  Every cell of
// cell_slots has its slot fixed by its own coordinates (row parity; column 0, or column parity), so
// the line's distinct (slot, cell) pairs are its distinct cells.  A line whose neighbours all lie in
// a 2x2 block of cells -- every line of an ordinary scan -- is counted with four warp min/max
// reductions and one OR of a 4-bit occupancy mask; any other line takes the slot analysis.
__device__ __forceinline__ int count_line_cells(float y, float x, int ny, int nx, bool periodic, uint32_t &err)
{
    Located L;
    const uint32_t e = locate(y, x, ny, nx, periodic, L);
    const int cy0 = L.iy0 >> 6, cy1 = L.iy1 >> 6;            // iy1 >= iy0
    const int cx0 = L.ix0 >> 6, cx1 = L.ix1 >> 6;            // cx1 < cx0 when x wraps
    // Most lines lie in one cell (a line is 32 samples, a cell 64 pixels wide): one pair, found with
    // a shuffle and a vote, as analyse_line does.
    const int c = (cy0 << 10) | cx0;
    const int c0 = __shfl_sync(kFullMask, c, 0);   // every lane takes part, before any short cut
    if (__all_sync(kFullMask, (cy0 == cy1) && (cx0 == cx1) && (c == c0))) {
        err |= e;
        return 1;
    }
    const int rmin = __reduce_min_sync(kFullMask, cy0);
    const int rmax = __reduce_max_sync(kFullMask, cy1);
    const int cmin = __reduce_min_sync(kFullMask, min(cx0, cx1));
    const int cmax = __reduce_max_sync(kFullMask, max(cx0, cx1));
    if ((rmax - rmin <= 1) && (cmax - cmin <= 1)) {
        err |= e;
        const int a0 = 2 * (cy0 - rmin), a1 = 2 * (cy1 - rmin);
        const int b0 = cx0 - cmin, b1 = cx1 - cmin;
        const unsigned m = (1u << (a0 + b0)) | (1u << (a0 + b1)) | (1u << (a1 + b0)) | (1u << (a1 + b1));
        return __popc(__reduce_or_sync(kFullMask, m));
    }
    LineSlots ls;
    return analyse_line(y, x, ny, nx, periodic, ls, err);
}

// Each planner block is counted by kPreplanSplit CTAs (a contiguous quarter of its lines each), which
// add their counts into the block's word: up to 1024 planner blocks would otherwise fill the GPU
// unevenly (about 1.4 waves).  nmt_out and err_out must be zero on entry.
constexpr int kPreplanSplit = 4;

__global__ void __launch_bounds__(kPlanWarps * 32)
preplan_count_kernel(const float *__restrict__ xp, int64_t nsamp, int ny, int nx, bool periodic,
                     int64_t nclpb, uint32_t *__restrict__ nmt_out, uint32_t *__restrict__ err_out)
{
    __shared__ uint32_t s_n[kPlanWarps];
    __shared__ uint32_t s_e[kPlanWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t ncl = nsamp >> 5;
    const int64_t pb = blockIdx.x / kPreplanSplit, part = blockIdx.x % kPreplanSplit;
    const int64_t b0 = pb * nclpb, b1 = min(ncl, b0 + nclpb);
    const int64_t chunk = (nclpb + kPreplanSplit - 1) / kPreplanSplit;
    const int64_t l0 = b0 + part * chunk;
    const int64_t l1 = min(b1, l0 + chunk);
    uint32_t n = 0, err = 0;

    for (int64_t lb = l0 + warp * kLinesPerWarp; lb < l1; lb += kRoundLines) {
        float y[kLinesPerWarp], x[kLinesPerWarp];
#pragma unroll
        for (int j = 0; j < kLinesPerWarp; j++) {
            int64_t l = min(lb + j, l1 - 1);
            y[j] = __ldcs(xp + 32 * l + lane);
            x[j] = __ldcs(xp + nsamp + 32 * l + lane);
        }
#pragma unroll
        for (int j = 0; j < kLinesPerWarp; j++) {
            if (lb + j >= l1)
                break;
            n += count_line_cells(y[j], x[j], ny, nx, periodic, err);
        }
    }

    err = __reduce_or_sync(kFullMask, err);
    if (lane == 0) {
        s_n[warp] = n;   // warp-uniform
        s_e[warp] = err;
    }
    __syncthreads();
    if (warp == 0) {
        uint32_t nn = (lane < kPlanWarps) ? s_n[lane] : 0u;
        uint32_t ee = (lane < kPlanWarps) ? s_e[lane] : 0u;
        nn = __reduce_add_sync(kFullMask, nn);
        ee = __reduce_or_sync(kFullMask, ee);
        if (lane == 0) {
            if (nn)
                atomicAdd(nmt_out + pb, nn);
            if (ee)
                atomicOr(err_out + pb, ee);
        }
    }
}

// Turns per-block counts into the inclusive cumsum padded with the total (PointingPrePlan.cu:203-211)
// and leaves {OR of error bits, total lo, total hi} in err[0..3) for one small readback.
__global__ void __launch_bounds__(1024)
preplan_finalize_kernel(uint32_t *__restrict__ nmt, uint32_t *__restrict__ err, int nblocks)
{
    __shared__ uint64_t s_w[32];
    __shared__ uint32_t s_e[32];
    __shared__ uint64_t s_total;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint64_t c = (t < nblocks) ? nmt[t] : 0;
    uint32_t e = (t < nblocks) ? err[t] : 0;
    uint64_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t v = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += v;
    }
    e = __reduce_or_sync(kFullMask, e);
    if (lane == 31) s_w[warp] = incl;
    if (lane == 0) s_e[warp] = e;
    __syncthreads();
    if (warp == 0) {
        const uint64_t w = s_w[lane];
        uint64_t wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint64_t v = __shfl_up_sync(kFullMask, wi, d);
            if (lane >= d) wi += v;
        }
        s_w[lane] = wi - w;
        const uint32_t ee = __reduce_or_sync(kFullMask, s_e[lane]);
        if (lane == 31) s_total = wi;
        if (lane == 0) s_e[0] = ee;
    }
    __syncthreads();
    incl += s_w[warp];
    const uint64_t total = s_total;   // blocks >= nblocks contribute 0
    nmt[t] = (uint32_t) ((t < nblocks) ? incl : total);
    if (t == 0) {
        err[0] = s_e[0];
        err[1] = (uint32_t) (total & 0xffffffffu);
        err[2] = (uint32_t) (total >> 32);
    }
}

// ------------------------------------------------------------------------------------------------
// Plan emit: deterministic, cache-line-major mt words per planner block, plus one owner word per
// cache line (the line's lowest cell), which the operators use to visit each line exactly once.

__global__ void __launch_bounds__(kPlanWarps * 32, 4)
plan_emit_kernel(const float *__restrict__ xp, int64_t nsamp, int ny, int nx, bool periodic, int64_t nclpb,
                 const uint32_t *__restrict__ nmt_cumsum, uint64_t *__restrict__ mt_out,
                 uint64_t *__restrict__ owner_out, uint64_t *__restrict__ band_out, uint32_t *__restrict__ errflags)
{
    __shared__ int s_cnt[kRoundLines];
    __shared__ int s_off[kRoundLines];
    __shared__ int s_fill[kRoundLines];
    __shared__ int s_ring[4];
    __shared__ int s_brow[kRoundLines];
    __shared__ int64_t s_base;
    // Slot analysis of each line of the round, kept here between the phases instead of in registers.
    __shared__ int s_slots[kRoundLines][6][32];
    __shared__ unsigned s_amask[kRoundLines][6];
    __shared__ uint32_t s_err[kPlanWarps];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t ncl = nsamp >> 5;
    const int64_t b = blockIdx.x;
    const int64_t l0 = b * nclpb;
    const int64_t l1 = min(ncl, l0 + nclpb);
    const int64_t out0 = b ? (int64_t) nmt_cumsum[b - 1] : 0;
    const int64_t nmax = (int64_t) nmt_cumsum[b] - out0;
    uint64_t *out = mt_out + out0;

    if (threadIdx.x < 4) s_ring[threadIdx.x] = 0;
    if (threadIdx.x == 0) s_base = 0;
    __syncthreads();

    uint32_t err = 0;

    for (int64_t r0 = l0; r0 < l1; r0 += kRoundLines) {
        // Phase 1: analyse this warp's lines of the round.
        float y[kLinesPerWarp], x[kLinesPerWarp];
        const int64_t lw = r0 + warp * kLinesPerWarp;
#pragma unroll
        for (int j = 0; j < kLinesPerWarp; j++) {
            int64_t l = min(lw + j, l1 - 1);
            y[j] = __ldcs(xp + 32 * l + lane);
            x[j] = __ldcs(xp + nsamp + 32 * l + lane);
        }
#pragma unroll
        for (int j = 0; j < kLinesPerWarp; j++) {
            int cnt = 0;
            LineSlots ls;
            if (lw + j < l1) {
                cnt = analyse_line(y[j], x[j], ny, nx, periodic, ls, err);
            } else {
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    ls.amask[k] = 0;
                    ls.slots[k] = -1;
                }
            }
            const int li = warp * kLinesPerWarp + j;
            // A line with one (cell, line) pair keeps only its cell (slot 0 at lane 0); the others
            // keep their whole slot analysis.
            if (cnt != 1) {
#pragma unroll
                for (int k = 0; k < 6; k++)
                    s_slots[li][k][lane] = ls.slots[k];
            }
            // Lowest upper footprint row of the line's samples (locate's clamp to [0, ny-2]).
            const int brow = __reduce_min_sync(kFullMask, min(max(__float2int_rz(y[j]), 0), ny - 2));
            if (lane == 0) {
                if (cnt != 1) {
#pragma unroll
                    for (int k = 0; k < 6; k++)
                        s_amask[li][k] = ls.amask[k];
                } else {
                    s_slots[li][0][0] = ls.slots[0];
                }
                s_cnt[li] = cnt;
                s_brow[li] = brow;
            }
        }
        __syncthreads();

        // Phase 2: offsets within the round and the reference's ring-buffer fill per line.
        // Line i of the round belongs to reference warp (i & 3) (PointingPlan.cu:167 with W=4;
        // r0 - l0 is a multiple of 32).
        if (warp == 0) {
            int c = s_cnt[lane];
            int incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                int v = __shfl_up_sync(kFullMask, incl, d);
                if (lane >= d) incl += v;
            }
            int cls = c;
#pragma unroll
            for (int d = 4; d < 32; d <<= 1) {
                int v = __shfl_up_sync(kFullMask, cls, d);
                if (lane >= d) cls += v;
            }
            s_off[lane] = incl - c;
            s_fill[lane] = (s_ring[lane & 3] + cls - c) & 31;
            int class_total = __shfl_sync(kFullMask, cls, 28 + (lane & 3));
            __syncwarp();
            if (lane < 4)
                s_ring[lane] = (s_ring[lane] + class_total) & 31;
        }
        __syncthreads();

        // Phase 3: emit.  Entry order within a line: slot order, then lane order (the order in
        // which the reference's ring buffer absorbs them, PointingPlan.cu:71-73, :182-187).
#pragma unroll
        for (int j = 0; j < kLinesPerWarp; j++) {
            const int li = warp * kLinesPerWarp + j;
            const int64_t l = r0 + li;
            if (l >= l1)
                break;
            const int64_t base = s_base + s_off[li];
            const int fill = s_fill[li];
            const int cnt = s_cnt[li];
            const bool mflag = (cnt > 1);
            const uint64_t hi = ((uint64_t) l << 20) | (mflag ? kMflag : 0ull);
            unsigned minc;
            if (cnt == 1) {
                // One word, at lane 0: no mflag, so no zflag.
                minc = (unsigned) s_slots[li][0][0];
                if ((lane == 0) && (base < nmax))
                    out[base] = (uint64_t) minc | hi;
            } else {
                int pos = 0;
                minc = 0xffffffffu;
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const unsigned am = s_amask[li][k];
                    if ((am >> lane) & 1u) {
                        const int rank = __popc(am & lt);
                        const int64_t p = base + pos + rank;
                        const bool zflag = mflag && (rank == 0) && (fill + pos < 32);
                        const int slot = s_slots[li][k][lane];
                        const uint64_t word = (uint64_t) (unsigned) slot | hi | (zflag ? kZflag : 0ull);
                        if (p < nmax)
                            out[p] = word;
                        minc = min(minc, (unsigned) slot);
                    }
                    pos += __popc(am);
                }
                minc = __reduce_min_sync(kFullMask, minc);
            }
            // Row band: the line's lowest row within the owner cell's rows, clamped to [0, 63].
            const int band = min(max(s_brow[li] - (int) ((minc >> 10) << 6), 0), 63);
            const uint64_t bw = band_line_word(y[j], x[j], (int) ((minc >> 10) << 6) + band, (int) ((minc & 1023u) << 6),
                                               ny, periodic ? (float) nx : (float) (nx - 2));
            if (lane == 0) {
                owner_out[l] = (uint64_t) minc | hi | ((uint64_t) band << kBandShift);
                band_out[l] = bw;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
            s_base += s_off[kRoundLines - 1] + s_cnt[kRoundLines - 1];
        __syncthreads();
    }

    if (s_base != nmax)
        err |= kErrInconsistentNmt;
    err = __reduce_or_sync(kFullMask, err);
    if (lane == 0)
        s_err[warp] = err;
    __syncthreads();
    if (warp == 0) {
        uint32_t e = (lane < kPlanWarps) ? s_err[lane] : 0u;
        e = __reduce_or_sync(kFullMask, e);
        if (lane == 0)
            errflags[b] = e;
    }
}

// ------------------------------------------------------------------------------------------------
// Hand-written stable LSD radix sort of mt words by cell.
//
// Only the cell bits that can vary are sorted: the compound key is ix | (iy << xbits), an order-
// preserving compression of the 20-bit cell field.  Each pass: upsweep (digit histogram per CTA
// chunk), a one-CTA exclusive scan, and a downsweep that ranks keys stably (warp match + per-warp
// running counts + a cross-warp scan per tile) and scatters them.

struct DigitSpec {
    int xbits;       // bits of the ixcell part
    uint32_t xmask;  // (1 << xbits) - 1
    uint32_t ymask;  // mask of the iycell part
    int ybits;       // bits of the iycell part
    uint32_t tmask;  // mask of the TOD index (bits 48+ of batch words) above the cell; 0: cell only
    uint32_t lmask;  // mask of the row band (bits 48+ of single-TOD owner words) below the cell; 0: none
    int lbits;       // bits of the row band part
    int shift;       // first compound bit of this pass
    int dbits;       // digit width of this pass
};

// Compound sort key of a word: band | (ixcell | iycell << xbits) << lbits | tod << (lbits + xbits + ybits),
// of which this pass takes 'dbits' bits from bit 'shift'.  A word has a band or a TOD index, not both.
__device__ __forceinline__ uint32_t key_digit(uint64_t w, const DigitSpec &ds)
{
    uint32_t c = (uint32_t) w;
    uint32_t ix = c & 0x3ffu, iy = (c >> 10) & 0x3ffu;
    const uint32_t hi = (uint32_t) (w >> 48);
    uint32_t comp = (hi & ds.lmask) | (((ix & ds.xmask) | ((iy & ds.ymask) << ds.xbits)) << ds.lbits) |
                    ((hi & ds.tmask) << (ds.lbits + ds.xbits + ds.ybits));
    return (comp >> ds.shift) & ((1u << ds.dbits) - 1u);
}

__global__ void __launch_bounds__(256)
sort_upsweep_kernel(const uint64_t *__restrict__ keys, int64_t n, int64_t chunk, DigitSpec ds,
                    uint32_t *__restrict__ hist)
{
    extern __shared__ uint32_t sh[];
    const int nd = 1 << ds.dbits;
    const int G = gridDim.x, g = blockIdx.x;
    const unsigned lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (int d = threadIdx.x; d < nd; d += blockDim.x)
        sh[d] = 0;
    __syncthreads();
    const int64_t c0 = g * chunk, c1 = min(n, c0 + chunk);
    for (int64_t i0 = c0; i0 < c1; i0 += blockDim.x) {
        const int64_t i = i0 + threadIdx.x;
        const bool valid = i < c1;
        const uint32_t d = valid ? key_digit(keys[i], ds) : 0xffffffffu;
        const unsigned peers = __match_any_sync(kFullMask, d);
        if (valid && ((peers & lt) == 0))
            atomicAdd(&sh[d], (uint32_t) __popc(peers));
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nd; d += blockDim.x)
        hist[(int64_t) d * G + g] = sh[d];
}

// Exclusive scan of hist[0..m) in place, one CTA of 1024 threads.
__global__ void __launch_bounds__(1024)
sort_scan_kernel(uint32_t *__restrict__ hist, int64_t m)
{
    __shared__ uint32_t s_w[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t seg = (m + 1023) / 1024;
    const int64_t a = min(m, t * seg), z = min(m, a + seg);
    uint32_t sum = 0;
    for (int64_t i = a; i < z; i++)
        sum += hist[i];
    uint32_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t v = __shfl_up_sync(kFullMask, incl, d);
        if (lane >= d) incl += v;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = s_w[lane], wi = w;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t v = __shfl_up_sync(kFullMask, wi, d);
            if (lane >= d) wi += v;
        }
        s_w[lane] = wi - w;
    }
    __syncthreads();
    uint32_t run = s_w[warp] + incl - sum;
    for (int64_t i = a; i < z; i++) {
        uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
}

constexpr int kSortWarps = 8;

template<int K>
__global__ void __launch_bounds__(kSortWarps * 32)
sort_downsweep_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out, int64_t n, int64_t chunk,
                      DigitSpec ds, const uint32_t *__restrict__ offs)
{
    extern __shared__ uint32_t sh[];
    const int nd = 1 << ds.dbits;
    uint32_t *whist = sh;                        // [kSortWarps][nd]
    uint32_t *run = sh + kSortWarps * nd;        // [nd]
    const int G = gridDim.x, g = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;

    for (int d = threadIdx.x; d < nd; d += blockDim.x)
        run[d] = offs[(int64_t) d * G + g];
    for (int i = threadIdx.x; i < kSortWarps * nd; i += blockDim.x)
        whist[i] = 0;
    __syncthreads();

    const int64_t c0 = g * chunk, c1 = min(n, c0 + chunk);
    constexpr int kTile = kSortWarps * 32 * K;
    uint32_t *mine = whist + warp * nd;

    for (int64_t t0 = c0; t0 < c1; t0 += kTile) {
        uint64_t key[K];
        uint32_t dig[K], rank[K];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int64_t i = t0 + (int64_t) warp * 32 * K + 32 * k + lane;
            const bool valid = i < c1;
            key[k] = valid ? in[i] : 0ull;
            dig[k] = valid ? key_digit(key[k], ds) : 0xffffffffu;
        }
#pragma unroll
        for (int k = 0; k < K; k++) {
            const bool valid = dig[k] != 0xffffffffu;
            const unsigned peers = __match_any_sync(kFullMask, dig[k]);
            const uint32_t prior = valid ? mine[dig[k]] : 0u;
            __syncwarp();
            if (valid && ((peers & lt) == 0))
                mine[dig[k]] = prior + __popc(peers);
            __syncwarp();
            rank[k] = prior + __popc(peers & lt);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < nd; d += blockDim.x) {
            uint32_t s = run[d];
#pragma unroll
            for (int w = 0; w < kSortWarps; w++) {
                uint32_t c = whist[w * nd + d];
                whist[w * nd + d] = s;
                s += c;
            }
            run[d] = s;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < K; k++)
            if (dig[k] != 0xffffffffu)
                out[mine[dig[k]] + rank[k]] = key[k];
        __syncthreads();
        for (int i = threadIdx.x; i < kSortWarps * nd; i += blockDim.x)
            whist[i] = 0;
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------------
// Cell bitmap of a sorted plan: one bit per cell that occurs in plan_mt.  The operators check it
// against the local pixelization, which gives the reference's not-in-pixelization semantics (an
// error iff the plan touches an absent cell, map2tod.cu:127-129) without any per-sample test.

__global__ void __launch_bounds__(256)
plan_cellmap_kernel(const uint64_t *__restrict__ plan_mt, int64_t nmt, uint32_t *__restrict__ cellmap)
{
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < nmt; i += stride) {
        const uint32_t c = (uint32_t) (plan_mt[i] & kCellMask);
        const uint32_t prev = (i > 0) ? (uint32_t) (plan_mt[i - 1] & kCellMask) : 0xffffffffu;
        if (c != prev)
            atomicOr(cellmap + (c >> 5), 1u << (c & 31));
    }
}

// ------------------------------------------------------------------------------------------------
// Dynamic-map cell discovery (expand_dynamic_map.cu:18-102): the last word of every cell run in
// the sorted plan is a candidate; targeted cells (offset -1) get the next free cell index.

__global__ void __launch_bounds__(256)
expand_dynamic_map_kernel(uint32_t *__restrict__ global_ncells, int64_t *__restrict__ cell_offsets, int nycells,
                          int nxcells, const uint64_t *__restrict__ plan_mt, int64_t nmt)
{
    __shared__ uint32_t s_cells[256];
    __shared__ uint32_t s_n, s_base;
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    const int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x;
    if (i < nmt) {
        const uint32_t c = (uint32_t) (plan_mt[i] & kCellMask);
        const uint32_t cn = (i + 1 < nmt) ? (uint32_t) (plan_mt[i + 1] & kCellMask) : 0xffffffffu;
        const uint32_t ix = c & 0x3ffu, iy = c >> 10;
        if ((c != cn) && (ix < (uint32_t) nxcells) && (iy < (uint32_t) nycells)) {
            if (cell_offsets[(int64_t) iy * nxcells + ix] == -1) {
                uint32_t k = atomicAdd(&s_n, 1u);
                s_cells[k] = c;
            }
        }
    }
    __syncthreads();
    const uint32_t nloc = s_n;
    if (nloc == 0)
        return;
    if (threadIdx.x == 0)
        s_base = atomicAdd(global_ncells, nloc);
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nloc; k += blockDim.x) {
        const uint32_t c = s_cells[k];
        const uint32_t ix = c & 0x3ffu, iy = c >> 10;
        cell_offsets[(int64_t) iy * nxcells + ix] = (int64_t) (s_base + k) * (3 * 64 * 64);
    }
}

// ------------------------------------------------------------------------------------------------
// Host launchers.

static int bits_for(int64_t n)   // bits needed for values in [0, n)
{
    int b = 0;
    while ((1ll << b) < n) b++;
    return b;
}

int sort_passes(int nycells_max, int nxcells_max, int max_digit_bits, int *digit_bits, int tod_bits)
{
    const int cb = bits_for(nxcells_max) + bits_for(nycells_max) + tod_bits;
    if (cb == 0) {
        *digit_bits = 0;
        return 0;
    }
    const int p = (cb + max_digit_bits - 1) / max_digit_bits;
    *digit_bits = (cb + p - 1) / p;
    return p;
}

int64_t sort_scratch_nbytes(int digit_bits, int grid)
{
    if (digit_bits <= 0) return 0;
    return ((int64_t) (1 << digit_bits) * grid * 4 + 127) & ~127ll;
}

// Grid of the sort kernels: ~4096 keys per CTA, at most two CTAs per SM and never more than 320
// (the histogram scratch is sized for 320 CTAs).
static int sort_grid(int64_t n, int num_sms)
{
    int64_t g = (n + 4095) / 4096;
    g = std::min<int64_t>(g, std::min<int64_t>(2 * (int64_t) num_sms, 320));
    return (int) std::max<int64_t>(g, 1);
}

int sort_grid_for(int64_t n) { return sort_grid(n, device_sm_count()); }

// Sorts 'n' mt words by cell (with tod_bits > 0: by (TOD, cell); with band_bits > 0: by (cell, row band)),
// stably.  The input is in 'a'; the result ends in 'a' if npasses is even and in 'b' if it is odd
// (callers place the input accordingly).
cudaError_t radix_sort_mt(uint64_t *a, uint64_t *b, int64_t n, int nycells_max, int nxcells_max, int digit_bits,
                          int npasses, uint32_t *hist, cudaStream_t stream, int tod_bits, int band_bits)
{
    if ((n <= 0) || (npasses == 0))
        return cudaSuccess;
    const int xbits = bits_for(nxcells_max), ybits = bits_for(nycells_max);
    const int kbits = xbits + ybits + tod_bits + band_bits;
    const int G = sort_grid_for(n);
    const int64_t chunk = (((n + G - 1) / G) + 255) / 256 * 256;
    constexpr int K = 8;
    static std::atomic<uint64_t> down_done{0}, up_done{0};
    cudaError_t e = set_smem_limit(sort_downsweep_kernel<K>, 200 * 1024, down_done);
    if (e == cudaSuccess)
        e = set_smem_limit(sort_upsweep_kernel, 64 * 1024, up_done);
    if (e != cudaSuccess)
        return e;
    uint64_t *src = a, *dst = b;
    for (int p = 0; p < npasses; p++) {
        DigitSpec ds;
        ds.xbits = xbits;
        ds.xmask = (1u << xbits) - 1u;
        ds.ymask = (1u << ybits) - 1u;
        ds.ybits = ybits;
        ds.tmask = (1u << tod_bits) - 1u;
        ds.lmask = (1u << band_bits) - 1u;
        ds.lbits = band_bits;
        ds.shift = p * digit_bits;
        ds.dbits = min(digit_bits, kbits - p * digit_bits);
        const int ndp = 1 << ds.dbits;
        sort_upsweep_kernel<<<G, 256, ndp * sizeof(uint32_t), stream>>>(src, n, chunk, ds, hist);
        sort_scan_kernel<<<1, 1024, 0, stream>>>(hist, (int64_t) ndp * G);
        sort_downsweep_kernel<K><<<G, kSortWarps * 32, (kSortWarps + 1) * ndp * sizeof(uint32_t), stream>>>(
            src, dst, n, chunk, ds, hist);
        uint64_t *t = src; src = dst; dst = t;
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Batch plan: one owner word per cache line of every TOD of a batch.

// Index of the TOD holding global cache line 'gl' (descs[i].line0 ascending): binary search.
__device__ __forceinline__ int batch_tod_of_line(const gmm_tod_desc *__restrict__ descs, int ntod, int64_t gl)
{
    int lo = 0, hi = ntod - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&descs[mid].line0) <= gl)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Marks 'cell' in the cell bitmap unless it is in this warp's cache of recently marked cells (one
// entry per lane 0..7, round robin); 'cell' is warp-uniform.
__device__ __forceinline__ void mark_cell(uint32_t cell, uint32_t tag, uint32_t *cellmap, uint32_t &cache, int &next)
{
    const int lane = threadIdx.x & 31;
    const uint32_t key = cell | tag;   // 'tag' distinguishes per-TOD bitmaps (0 for one shared bitmap)
    if (__ballot_sync(kFullMask, (lane < 8) && (cache == key)) != 0u)
        return;
    if (lane == 0)
        atomicOr(cellmap + (cell >> 5), 1u << (cell & 31));
    if (lane == next)
        cache = key;
    next = (next + 1) & 7;
}

// Cell bitmap of a single-TOD batch plan buffer: after its nlines owner words, 128-byte aligned.
__device__ __forceinline__ uint32_t *single_plan_cellmap(void *plan, int64_t nlines)
{
    return (uint32_t *) ((char *) plan + ((8 * nlines + 127) & ~127ll));
}

// One warp per cache line (lane = sample).  Each CTA takes a contiguous range of the batch's lines
// and its warps interleave over it, so a warp sees nearby pointing and its cache of marked cells
// keeps the bitmap atomics to about one per cell and warp.  The owner cell is the lowest cell
// among the four neighbours of the line's samples (the cells of a line are those of
// cell_enumerator, gpu_mm_internals.hpp:179-237); every cell the line touches is marked in the
// cell bitmap.  Word = cell | line << 20 | mflag << 46 | tod << 48, at the line's global index.
__global__ void __launch_bounds__(256)
batch_owner_kernel(const gmm_tod_desc *__restrict__ descs, int ntod, int64_t total_lines, int ny, int nx,
                   bool periodic, uint64_t *__restrict__ owner_out, uint32_t *__restrict__ cellmap,
                   void *const *__restrict__ plans_each, uint32_t *__restrict__ errword)
{
    // plans_each (optional): per-TOD single-TOD plan buffers whose own cell bitmaps are marked
    // instead of the shared 'cellmap'.
    __shared__ uint32_t s_err[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t l0 = (total_lines * (int64_t) blockIdx.x) / gridDim.x;
    const int64_t l1 = (total_lines * (int64_t) (blockIdx.x + 1)) / gridDim.x;
    uint32_t err = 0;
    uint32_t cache = 0xffffffffu;   // no cell id is all ones
    int next = 0;
    for (int64_t gl = l0 + warp; gl < l1; gl += nw) {
        const int tod = batch_tod_of_line(descs, ntod, gl);
        const float *xp = (const float *) __ldg((const unsigned long long *) &descs[tod].xpointing);
        const int64_t nsamp = __ldg(&descs[tod].nsamp);
        const int64_t line = gl - __ldg(&descs[tod].line0);
        // Descriptors that do not match total_lines (line outside its TOD) are flagged; the line's
        // word carries bit 47 ("invalid"), which the operators refuse.
        if ((line < 0) || (32 * line >= nsamp) || (line >= (1ll << 26))) {
            err |= kErrInconsistentNmt;
            if (lane == 0)
                owner_out[gl] = kZflag | ((uint64_t) tod << kBatchTodShift);
            continue;
        }
        const int64_t s = 32 * line + lane;
        Located L;
        err |= locate(__ldcs(xp + s), __ldcs(xp + nsamp + s), ny, nx, periodic, L);
        const uint32_t c[4] = {((uint32_t) (L.iy0 >> 6) << 10) | (uint32_t) (L.ix0 >> 6),
                               ((uint32_t) (L.iy0 >> 6) << 10) | (uint32_t) (L.ix1 >> 6),
                               ((uint32_t) (L.iy1 >> 6) << 10) | (uint32_t) (L.ix0 >> 6),
                               ((uint32_t) (L.iy1 >> 6) << 10) | (uint32_t) (L.ix1 >> 6)};
        const uint32_t lo = min(min(c[0], c[1]), min(c[2], c[3]));
        const uint32_t hi = max(max(c[0], c[1]), max(c[2], c[3]));
        const uint32_t owner = __reduce_min_sync(kFullMask, lo);
        const bool multi = __any_sync(kFullMask, hi != owner);
        if (lane == 0)
            owner_out[gl] = (uint64_t) owner | ((uint64_t) line << 20) | ((uint64_t) multi << 46) |
                            ((uint64_t) tod << kBatchTodShift);
        uint32_t *cm = cellmap;
        uint32_t tag = 0;
        if (plans_each) {
            cm = single_plan_cellmap(plans_each[tod], nsamp >> 5);
            tag = ((uint32_t) tod & 0xfffu) << 20;
        }
        mark_cell(owner, tag, cm, cache, next);
        if (multi) {
            // The line's other cells: one representative lane per distinct value of each corner.
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const unsigned peers = __match_any_sync(kFullMask, c[k]);
                unsigned lead = __ballot_sync(kFullMask, ((peers & ((1u << lane) - 1u)) == 0u) && (c[k] != owner));
                while (lead) {
                    const int src = __ffs(lead) - 1;
                    lead &= lead - 1;
                    mark_cell(__shfl_sync(kFullMask, c[k], src), tag, cm, cache, next);
                }
            }
        }
    }
    err = __reduce_or_sync(kFullMask, err);
    if (lane == 0)
        s_err[warp] = err;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t e = 0;
        for (int w = 0; w < nw; w++)
            e |= s_err[w];
        if (e)
            atomicOr(errword, e);
    }
}

// Merge of single-TOD batch plans: CTA b of the grid copies TOD (b % ntod)'s owner words with the
// TOD index set, grid-striding over that TOD; destination offsets are the prefix sums of nlines.
__global__ void __launch_bounds__(256)
batch_merge_kernel(const void *const *__restrict__ plans, const int64_t *__restrict__ nlines, int ntod,
                   uint64_t *__restrict__ owner_out, uint32_t *__restrict__ cellmap)
{
    __shared__ int64_t s_off;
    const int tod = blockIdx.x % ntod;
    const int part = blockIdx.x / ntod, nparts = gridDim.x / ntod;
    if (threadIdx.x == 0) {
        int64_t off = 0;
        for (int i = 0; i < tod; i++)
            off += nlines[i];
        s_off = off;
    }
    __syncthreads();
    const int64_t n = nlines[tod];
    const uint64_t *src = (const uint64_t *) plans[tod];
    const uint64_t tag = (uint64_t) tod << kBatchTodShift;
    for (int64_t k = part * (int64_t) blockDim.x + threadIdx.x; k < n; k += (int64_t) nparts * blockDim.x)
        owner_out[s_off + k] = (src[k] & ((1ull << kBatchTodShift) - 1)) | tag;
    // A single-TOD plan holds its n owner words, then (128-byte aligned) its cell bitmap.
    const uint32_t *cm = (const uint32_t *) ((const char *) plans[tod] + ((8 * n + 127) & ~127ll));
    for (int w = part * blockDim.x + threadIdx.x; w < (1 << 15); w += nparts * blockDim.x) {
        const uint32_t bits = cm[w];
        if (bits)
            atomicOr(cellmap + w, bits);
    }
}

cudaError_t launch_batch_merge(const void *const *plans, const int64_t *nlines, int ntod, int64_t total_lines,
                               uint64_t *owner_out, uint32_t *cellmap, cudaStream_t stream)
{
    if (ntod <= 0)
        return cudaSuccess;
    const int64_t per_tod = std::max<int64_t>(1, std::min<int64_t>(64, (total_lines / ntod + 4095) / 4096));
    batch_merge_kernel<<<(unsigned) (per_tod * ntod), 256, 0, stream>>>(plans, nlines, ntod, owner_out, cellmap);
    return cudaGetLastError();
}

cudaError_t launch_batch_owner(const gmm_tod_desc *descs, int ntod, int64_t total_lines, int ny, int nx, bool periodic,
                               uint64_t *owner_out, uint32_t *cellmap, void *const *plans_each, uint32_t *errword,
                               cudaStream_t stream)
{
    if (total_lines <= 0)
        return cudaSuccess;
    // Contiguous ranges of >= 256 lines per CTA (8 warps).
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((total_lines + 255) / 256, 8 * (int64_t) device_sm_count()));
    batch_owner_kernel<<<(unsigned) g, 256, 0, stream>>>(descs, ntod, total_lines, ny, nx, periodic, owner_out, cellmap,
                                                         plans_each, errword);
    return cudaGetLastError();
}

// Building many single-TOD plans at once: clear their cell bitmaps, then (after the owner kernel and
// a sort by (TOD, cell)) copy TOD i's segment [line0_i, line0_i + nlines_i) into its own buffer.
__global__ void __launch_bounds__(256)
clear_cellmaps_kernel(const gmm_tod_desc *__restrict__ descs, int ntod, void *const *__restrict__ plans)
{
    const int tod = blockIdx.x % ntod, part = blockIdx.x / ntod, nparts = gridDim.x / ntod;
    uint32_t *cm = single_plan_cellmap(plans[tod], __ldg(&descs[tod].nsamp) >> 5);
    for (int w = part * blockDim.x + threadIdx.x; w < (1 << 15); w += nparts * blockDim.x)
        cm[w] = 0u;
}

__global__ void __launch_bounds__(256)
scatter_each_kernel(const gmm_tod_desc *__restrict__ descs, const uint64_t *__restrict__ sorted, int64_t total_lines,
                    void *const *__restrict__ plans)
{
    for (int64_t p = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; p < total_lines;
         p += (int64_t) gridDim.x * blockDim.x) {
        const uint64_t w = sorted[p];
        const int tod = (int) (w >> kBatchTodShift);
        // With consistent descriptors TOD i's entries are exactly [line0_i, line0_i + nlines_i);
        // anything else (already flagged by the owner kernel) is not written.
        const int64_t k = p - __ldg(&descs[tod].line0);
        if ((k >= 0) && (k < (__ldg(&descs[tod].nsamp) >> 5)))
            ((uint64_t *) plans[tod])[k] = w & ((1ull << kBatchTodShift) - 1);
    }
}

cudaError_t launch_plans_each(const gmm_tod_desc *descs, int ntod, int64_t total_lines, int ny, int nx, bool periodic,
                              void *const *plans, uint64_t *a, uint64_t *b, uint32_t *hist, int digit_bits,
                              int npasses, int tod_bits, uint32_t *errword, cudaStream_t stream)
{
    if (total_lines <= 0)
        return cudaSuccess;
    const int nyc = (ny + 63) / 64, nxc = (nx + 63) / 64;
    clear_cellmaps_kernel<<<(unsigned) (ntod * 4), 256, 0, stream>>>(descs, ntod, plans);
    cudaError_t e = launch_batch_owner(descs, ntod, total_lines, ny, nx, periodic, a, nullptr, plans, errword, stream);
    if (e == cudaSuccess)
        e = radix_sort_mt(a, b, total_lines, nyc, nxc, digit_bits, npasses, hist, stream, tod_bits);
    if (e != cudaSuccess)
        return e;
    const uint64_t *sorted = (npasses % 2 == 0) ? a : b;
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((total_lines + 255) / 256, 8 * (int64_t) device_sm_count()));
    scatter_each_kernel<<<(unsigned) g, 256, 0, stream>>>(descs, sorted, total_lines, plans);
    return cudaGetLastError();
}

cudaError_t launch_preplan(const float *xp, int64_t nsamp, int ny, int nx, bool periodic, int64_t nclpb,
                           int nblocks, uint32_t *nmt, uint32_t *err, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(nmt, 0, (size_t) nblocks * sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(err, 0, (size_t) nblocks * sizeof(uint32_t), stream);
    if (e != cudaSuccess)
        return e;
    preplan_count_kernel<<<(unsigned) nblocks * kPreplanSplit, kPlanWarps * 32, 0, stream>>>(xp, nsamp, ny, nx,
                                                                                           periodic, nclpb, nmt, err);
    preplan_finalize_kernel<<<1, 1024, 0, stream>>>(nmt, err, nblocks);
    return cudaGetLastError();
}

cudaError_t launch_plan_emit(const float *xp, int64_t nsamp, int ny, int nx, bool periodic, int64_t nclpb,
                             int nblocks, const uint32_t *nmt_cumsum, uint64_t *mt_out, uint64_t *owner_out,
                             uint64_t *band_out, uint32_t *errflags, cudaStream_t stream)
{
    plan_emit_kernel<<<nblocks, kPlanWarps * 32, 0, stream>>>(xp, nsamp, ny, nx, periodic, nclpb, nmt_cumsum,
                                                               mt_out, owner_out, band_out, errflags);
    return cudaGetLastError();
}

// Band words into owner-list order: band_out[q] = band_by_line[line of owner[q]].
__global__ void __launch_bounds__(256)
band_gather_kernel(const uint64_t *__restrict__ owner, int64_t n, const uint64_t *__restrict__ band_by_line,
                   uint64_t *__restrict__ band_out)
{
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t q = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; q < n; q += stride)
        band_out[q] = band_by_line[(owner[q] >> 20) & kClMask];
}

cudaError_t launch_band_gather(const uint64_t *owner, int64_t n, const uint64_t *band_by_line, uint64_t *band_out,
                               cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8 * (int64_t) device_sm_count()));
    band_gather_kernel<<<(unsigned) g, 256, 0, stream>>>(owner, n, band_by_line, band_out);
    return cudaGetLastError();
}

cudaError_t launch_plan_cellmap(const uint64_t *plan_mt, int64_t nmt, uint32_t *cellmap, cudaStream_t stream)
{
    if (nmt <= 0)
        return cudaSuccess;
    const int64_t g = std::min<int64_t>((nmt + 255) / 256, 8 * (int64_t) device_sm_count());
    plan_cellmap_kernel<<<(unsigned) g, 256, 0, stream>>>(plan_mt, nmt, cellmap);
    return cudaGetLastError();
}

cudaError_t launch_expand_dynamic_map(uint32_t *global_ncells, int64_t *cell_offsets, int nycells, int nxcells,
                                      const uint64_t *plan_mt, int64_t nmt, cudaStream_t stream)
{
    if (nmt <= 0)
        return cudaSuccess;
    const int64_t nb = (nmt + 255) / 256;
    expand_dynamic_map_kernel<<<(unsigned) nb, 256, 0, stream>>>(global_ncells, cell_offsets, nycells, nxcells,
                                                                  plan_mt, nmt);
    return cudaGetLastError();
}

}  // namespace gmm
