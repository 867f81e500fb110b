// Pointing operators on sm_100a: planned and unplanned map2tod / tod2map (+ response variants).
//
// Semantics follow the reference CPU operators (kmsmith137/gpu_mm src_lib/map2tod_reference.cu:16-54,
// tod2map_reference.cu:14-46) and the planned GPU ones (map2tod.cu, tod2map.cu, map2tod_response.cu,
// tod2map_response.cu): bilinear T/Q/U interpolation with the cos 2a / sin 2a response, cells of
// 64x64 pixels addressed through cell_offsets, and x-wraparound.
//
// Planned design (this implementation's own):
//  * Every 32-sample cache line is processed exactly once, by the CTA that holds its "owner" cell
//    (the lowest cell the line touches).  The plan carries that owner list sorted by cell; a CTA
//    walks a contiguous slice of it.  Its warps walk the slice independently and meet at a barrier
//    only when the cell changes, which is when the tile is reloaded (map2tod) or flushed (tod2map).
//  * The tile is the owner cell plus a halo: rows [0, 64+HY) and columns [-HX, 64+HX) around the
//    cell, in unwrapped x.  A line's whole bilinear footprint normally fits, so no cache line is
//    read twice, no TOD word needs an atomic, and no pre-zeroing pass is needed.  Samples that do
//    not fit take an exact path through global memory.
//  * Absent cells read as zero.  The not-in-pixelization error is decided per plan cell (the plan
//    carries a bitmap of its cells), exactly the reference's condition, so the sample loop does no
//    presence test.
//  * tod2map accumulates into the tile with shared-memory atomics.  Adjacent samples usually hit
//    the same pixel, so lane i adds T, Q and U in an order rotated by i mod 3: in one atomic
//    instruction, neighbouring lanes then target different words.
//  * With the plain float flush, only the upper row of a sample's 2x2 footprint goes into the tile;
//    the lower row is added straight into the map with fire-and-forget reductions, which the L2
//    executes.  Shared-memory float atomics are compare-and-swap loops on this GPU and were the
//    bound; splitting the footprint puts half of the work on each unit, which run in parallel.
//  * xpointing and TOD are streamed with evict-first loads/stores so that the map and plan stay in
//    L2; each warp keeps UNR cache lines in flight.
#include <algorithm>

#include "gmm_internal.hpp"

namespace gmm {

int g_tod2map_kernel = GMM_TOD2MAP_BANDS;

namespace {

constexpr int HX = 32;                 // halo columns on each side
constexpr int HY = 4;                  // halo rows below the cell
constexpr int TY = 64 + HY;            // tile rows
constexpr int TX = 64 + 2 * HX;        // tile columns
constexpr int TS = TX + 1;             // padded row stride in shared memory
constexpr int PS = TY * TS;            // one polarisation plane
constexpr int NW = 16;                 // warps per CTA
constexpr int NT = NW * 32;
constexpr int UNR = 4;                 // cache lines in flight per warp
constexpr int CH = 4;                  // owner entries a warp decodes at once (a multiple of UNR)
constexpr size_t kTileBytes = 3 * (size_t) PS * sizeof(float);
constexpr int kCellmapWords = (1 << 20) / 32;

struct Tile {
    int gy0;   // global row of tile row 0
    int gx0;   // unwrapped global column of tile column 0
};

// Per-tile offset table, computed once per tile: tab[b * TX + c] is the local-map offset of tile
// column c in row 0 of row block b (tile rows [64b, 64b + 64), all in one cell row), or -1 if that
// column is outside the map or its cell is absent.  Tile pixel (r, c) is then at
// tab[(r / 64) * TX + c] + (r % 64) * ystride, so the tile loops issue their map loads with no
// cell_offsets lookup in between.
constexpr int kTabEntries = 2 * TX;

__device__ void tile_offsets(int64_t *tab, const Tile &T, const OpArgs &a)
{
    for (int i = threadIdx.x; i < kTabEntries; i += blockDim.x) {
        const int b = i / TX, c = i % TX;
        const int cy = (T.gy0 >> 6) + b;
        int gx = T.gx0 + c;
        if (a.periodic) {
            gx %= a.nx;
            gx += (gx < 0) ? a.nx : 0;
        }
        int64_t off = -1;
        if ((gx >= 0) && (cy < a.nycells) && (gx < 64 * a.nxcells)) {
            const int64_t co = __ldg(a.cell_offsets + (int64_t) cy * a.nxcells + (gx >> 6));
            off = (co >= 0) ? (co + (gx & 63)) : -1;
        }
        tab[i] = off;
    }
}

// cp.async of 16 bytes, global -> shared (L2 only), and its group bookkeeping.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const uint32_t d = (uint32_t) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template<int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Global-memory pixel offset (map_evaluator / map_accumulator addressing,
// gpu_mm_internals.hpp:258-275), or -1 if the cell is absent.
__device__ __forceinline__ int64_t global_pixel_offset(int iy, int ix, const OpArgs &a)
{
    const int iyc = iy >> 6, ixc = ix >> 6;
    if ((iyc >= a.nycells) || (ixc >= a.nxcells))
        return -1;
    const int64_t off = __ldg(a.cell_offsets + (int64_t) iyc * a.nxcells + ixc);
    if (off < 0)
        return -1;
    return off + (int64_t) (iy & 63) * a.ystride + (ix & 63);
}

__device__ __forceinline__ uint32_t detector_of(const OpArgs &a, uint32_t s)
{
    const uint32_t t = __umulhi(a.det_m, s);
    return (t + ((s - t) >> a.det_sh1)) >> a.det_sh2;
}

// Per-sample response factors (t_resp, p_resp) = (response[det], response[det+ndet])
// (map2tod_response.cu:168-176).
__device__ __forceinline__ void sample_response(const OpArgs &a, uint32_t s, float &tr, float &pr)
{
    const uint32_t det = detector_of(a, s);
    tr = __ldg(a.response + det);
    pr = __ldg(a.response + det + a.ndet);
}

// Loads the tile from the local map (absent pixels read as zero).  'tab' must hold the tile's
// offset table (tile_offsets) and be visible to all threads.  Pixels move in groups of four
// columns: a group whose four map pixels are consecutive and 16-byte aligned (the usual case: cell
// offsets, ystride and polstride multiples of 4) is read with one float4 load per plane, so a
// thread has all of its loads in flight at once; other groups are read pixel by pixel.
__device__ void load_tile(float *tile, const int64_t *tab, const OpArgs &a, const float *__restrict__ lmap)
{
    constexpr int NG = TY * (TX / 4);   // column groups
    const bool vec_ok = ((((uintptr_t) lmap) & 15) == 0) && ((a.ystride & 3) == 0) && ((a.polstride & 3) == 0);
#pragma unroll 4
    for (int gi = threadIdx.x; gi < NG; gi += blockDim.x) {
        const int r = gi / (TX / 4), c = 4 * (gi % (TX / 4));
        const int64_t *tb = tab + (r >> 6) * TX + c;
        const int64_t b0 = tb[0];
        const int64_t roff = (int64_t) (r & 63) * a.ystride;
        float *dst = tile + r * TS + c;
        if (vec_ok && (b0 >= 0) && ((b0 & 3) == 0) && (tb[1] == b0 + 1) && (tb[2] == b0 + 2) && (tb[3] == b0 + 3)) {
            const float4 *src = reinterpret_cast<const float4 *>(lmap + b0 + roff);
            const float4 t = __ldg(src);
            const float4 q = __ldg(src + a.polstride / 4);
            const float4 u = __ldg(src + a.polstride / 2);
            dst[0] = t.x; dst[1] = t.y; dst[2] = t.z; dst[3] = t.w;
            dst[PS] = q.x; dst[PS + 1] = q.y; dst[PS + 2] = q.z; dst[PS + 3] = q.w;
            dst[2 * PS] = u.x; dst[2 * PS + 1] = u.y; dst[2 * PS + 2] = u.z; dst[2 * PS + 3] = u.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int64_t bk = tb[k];
                const bool p = bk >= 0;
                const int64_t off = bk + roff;
                dst[k] = p ? __ldg(lmap + off) : 0.0f;
                dst[PS + k] = p ? __ldg(lmap + off + a.polstride) : 0.0f;
                dst[2 * PS + k] = p ? __ldg(lmap + off + 2 * a.polstride) : 0.0f;
            }
        }
    }
}

// One addition into the map at element 'off' in flush mode FLUSH (OpArgs::flush).  The
// compensated mode keeps the rounding error of each float atomic (Knuth's two-sum, from the old
// value the atomic returns) in 'comp', so that map + comp carries the sum to about twice float
// precision until gmm_fold_compensation folds it in.
// Rounding error of the float addition old + v (Knuth's two-sum), added into 'comp'.
__device__ __forceinline__ void add_rounding_error(const OpArgs &a, int64_t off, float old, float v)
{
    const float sum = __fadd_rn(old, v);
    const float bv = __fsub_rn(sum, old);
    const float e = __fadd_rn(__fsub_rn(old, __fsub_rn(sum, bv)), __fsub_rn(v, bv));
    if (e != 0.0f)
        atomicAdd(a.comp + off, e);
}

template<int FLUSH>
__device__ __forceinline__ void global_add(const OpArgs &a, int64_t off, float v)
{
    if constexpr (FLUSH == kFlushF64) {
        atomicAdd(a.out64 + off, (double) v);
    } else if constexpr (FLUSH == kFlushCompensated) {
        add_rounding_error(a, off, atomicAdd(a.out + off, v), v);
    } else {
        atomicAdd(a.out + off, v);
    }
}

// Flush mode kFlushHotF64: adds (t, q, u) at pixel (iy, ix) (inside the map) into the float64
// accumulator of the pixel's cell if the cell has a hot slot, else into the float map with float
// atomics (nothing for an absent cell).  Zeros are skipped.
__device__ __forceinline__ void hot_add3(const OpArgs &a, int iy, int ix, float t, float q, float u)
{
    const int iyc = iy >> 6, ixc = ix >> 6;
    if ((iyc >= a.nycells) || (ixc >= a.nxcells))
        return;
    const int64_t c = (int64_t) iyc * a.nxcells + ixc;
    const int slot = __ldg(a.hot_slot + c);
    if (slot >= 0) {
        double *h = a.hot + (int64_t) slot * kHotCellDoubles + (iy & 63) * 64 + (ix & 63);
        if (t != 0.0f) atomicAdd(h, (double) t);
        if (q != 0.0f) atomicAdd(h + 4096, (double) q);
        if (u != 0.0f) atomicAdd(h + 8192, (double) u);
        return;
    }
    const int64_t base = __ldg(a.cell_offsets + c);
    if (base < 0)
        return;
    float *m = a.out + base + (int64_t) (iy & 63) * a.ystride + (ix & 63);
    if (t != 0.0f) atomicAdd(m, t);
    if (q != 0.0f) atomicAdd(m + a.polstride, q);
    if (u != 0.0f) atomicAdd(m + 2 * a.polstride, u);
}

// Adds the tile into the map (one atomic per non-zero pixel and polarisation, in flush mode FLUSH)
// and clears it.
template<int FLUSH = kFlushF32>
__device__ void flush_tile(float *tile, const int64_t *tab, const OpArgs &a, float *__restrict__ lmap)
{
    for (int idx = threadIdx.x; idx < TY * TX; idx += NT) {
        const int r = idx / TX, c = idx % TX;
        float *src = tile + r * TS + c;
        const float t = src[0], q = src[PS], u = src[2 * PS];
        if ((t != 0.0f) || (q != 0.0f) || (u != 0.0f)) {
            const int64_t base = tab[(r >> 6) * TX + c];
            if (base >= 0) {
                const int64_t off = base + (int64_t) (r & 63) * a.ystride;
                if constexpr (FLUSH == kFlushF32) {
                    atomicAdd(lmap + off, t);
                    atomicAdd(lmap + off + a.polstride, q);
                    atomicAdd(lmap + off + 2 * a.polstride, u);
                } else if constexpr (FLUSH == kFlushCompensated) {
                    // The three returning atomics are issued before any result is used, so their
                    // round trips overlap.
                    const float ot = atomicAdd(lmap + off, t);
                    const float oq = atomicAdd(lmap + off + a.polstride, q);
                    const float ou = atomicAdd(lmap + off + 2 * a.polstride, u);
                    add_rounding_error(a, off, ot, t);
                    add_rounding_error(a, off + a.polstride, oq, q);
                    add_rounding_error(a, off + 2 * a.polstride, ou, u);
                } else {
                    global_add<FLUSH>(a, off, t);
                    global_add<FLUSH>(a, off + a.polstride, q);
                    global_add<FLUSH>(a, off + 2 * a.polstride, u);
                }
            }
            src[0] = 0.0f;
            src[PS] = 0.0f;
            src[2 * PS] = 0.0f;
        }
    }
}

// Position of a located sample inside the tile; false if its footprint is not inside.
template<bool PERIODIC>
__device__ __forceinline__ bool tile_position(const Located &L, const Tile &T, const OpArgs &a, int &ry, int &rx)
{
    ry = L.iy0 - T.gy0;
    rx = L.ix0 - T.gx0;
    if constexpr (PERIODIC) {
        rx += (rx < 0) ? a.nx : 0;
        rx -= (rx > TX - 2) ? a.nx : 0;
    }
    return ((unsigned) ry <= (unsigned) (TY - 2)) && ((unsigned) rx <= (unsigned) (TX - 2));
}

// The map2tod arithmetic of one sample, written with explicit round-to-nearest operations so that
// the compiler cannot contract it differently in different kernels: every path (fast or general,
// single TOD or batch, any grid) then gives the same bits for the same sample.
//   pol_eval: ct*T + cq*Q + cu*U (ct = 1 without a response, so T enters unscaled);
//   bilinear: (1-dy)(1-dx) e00 + (1-dy) dx e01 + dy (1-dx) e10 + dy dx e11, in that order.
template<bool RESP>
__device__ __forceinline__ float pol_eval(float ct, float cq, float cu, float t, float q, float u)
{
    return __fmaf_rn(cu, u, __fmaf_rn(cq, q, RESP ? __fmul_rn(ct, t) : t));
}

__device__ __forceinline__ float bilinear(float dy, float dx, float e00, float e01, float e10, float e11)
{
    const float wy0 = __fsub_rn(1.0f, dy), wx0 = __fsub_rn(1.0f, dx);
    float r = __fmul_rn(__fmul_rn(wy0, wx0), e00);
    r = __fmaf_rn(__fmul_rn(wy0, dx), e01, r);
    r = __fmaf_rn(__fmul_rn(dy, wx0), e10, r);
    return __fmaf_rn(__fmul_rn(dy, dx), e11, r);
}

template<bool RESP = false>
__device__ __forceinline__ float global_eval(const OpArgs &a, const float *__restrict__ lmap, int iy, int ix,
                                             float ct, float cq, float cu, uint32_t &err)
{
    const int64_t off = global_pixel_offset(iy, ix, a);
    const bool valid = off >= 0;
    const float t = valid ? __ldg(lmap + off) : 0.0f;
    const float q = valid ? __ldg(lmap + off + a.polstride) : 0.0f;
    const float u = valid ? __ldg(lmap + off + 2 * a.polstride) : 0.0f;
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
    return pol_eval<RESP>(ct, cq, cu, t, q, u);
}

// Local-map offsets (plane T) of a located sample's four neighbours, in the order (iy0, ix0),
// (iy0, ix1), (iy1, ix0), (iy1, ix1), or -1 where a neighbour is outside the map or in an absent
// cell: global_pixel_offset of each, with one cell_offsets lookup when all four lie in one cell and
// ix1 = ix0 + 1 (every footprint except those on a cell edge or across the x wrap-around).
__device__ __forceinline__ void neighbour_offsets(const Located &L, const OpArgs &a, int64_t off[4])
{
    const int cy = L.iy0 >> 6, cx = L.ix0 >> 6;
    if (((L.iy1 >> 6) == cy) && ((L.ix1 >> 6) == cx) && (L.ix1 == L.ix0 + 1)) {
        int64_t base = -1;
        if ((cy < a.nycells) && (cx < a.nxcells))
            base = __ldg(a.cell_offsets + (int64_t) cy * a.nxcells + cx);
        const int64_t o = base + (int64_t) (L.iy0 & 63) * a.ystride + (L.ix0 & 63);
        const bool in = base >= 0;
        off[0] = in ? o : -1;
        off[1] = in ? o + 1 : -1;
        off[2] = in ? o + a.ystride : -1;
        off[3] = in ? o + a.ystride + 1 : -1;
    } else {
        off[0] = global_pixel_offset(L.iy0, L.ix0, a);
        off[1] = global_pixel_offset(L.iy0, L.ix1, a);
        off[2] = global_pixel_offset(L.iy1, L.ix0, a);
        off[3] = global_pixel_offset(L.iy1, L.ix1, a);
    }
}

// global_eval without a response at a neighbour offset from neighbour_offsets (the same loads,
// error bit and arithmetic).
__device__ __forceinline__ float eval_at(const OpArgs &a, const float *__restrict__ lmap, int64_t off, float cq,
                                         float cu, uint32_t &err)
{
    const bool valid = off >= 0;
    const float t = valid ? __ldg(lmap + off) : 0.0f;
    const float q = valid ? __ldg(lmap + off + a.polstride) : 0.0f;
    const float u = valid ? __ldg(lmap + off + 2 * a.polstride) : 0.0f;
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
    return pol_eval<false>(1.0f, cq, cu, t, q, u);
}

template<int FLUSH = kFlushF32>
__device__ __forceinline__ void global_accum(const OpArgs &a, float *__restrict__ lmap, int iy, int ix,
                                             float t, float q, float u, float w, uint32_t &err)
{
    const int64_t off = global_pixel_offset(iy, ix, a);
    const bool valid = off >= 0;
    if (valid) {
        if constexpr (FLUSH == kFlushF32) {
            atomicAdd(lmap + off, w * t);
            atomicAdd(lmap + off + a.polstride, w * q);
            atomicAdd(lmap + off + 2 * a.polstride, w * u);
        } else {
            global_add<FLUSH>(a, off, w * t);
            global_add<FLUSH>(a, off + a.polstride, w * q);
            global_add<FLUSH>(a, off + 2 * a.polstride, w * u);
        }
    }
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
}

// Bilinear map2tod value of a sample at tile offset p: sum over the four neighbours of weight x
// (ct*T + cq*Q + cu*U) (map_evaluator, gpu_mm_internals.hpp:243-293, on the staged tile).
template<bool RESP>
__device__ __forceinline__ float tile_eval(const float *tile, int p, float ct, float cq, float cu, float dy, float dx)
{
    const float *q = tile + p;
    const float e00 = pol_eval<RESP>(ct, cq, cu, q[0], q[PS], q[2 * PS]);
    const float e01 = pol_eval<RESP>(ct, cq, cu, q[1], q[PS + 1], q[2 * PS + 1]);
    const float e10 = pol_eval<RESP>(ct, cq, cu, q[TS], q[PS + TS], q[2 * PS + TS]);
    const float e11 = pol_eval<RESP>(ct, cq, cu, q[TS + 1], q[PS + TS + 1], q[2 * PS + TS + 1]);
    return bilinear(dy, dx, e00, e01, e10, e11);
}

// tile_eval without a response for two samples at tile offsets p0, p1, with packed float pairs: the
// same operations in the same order, so the same bits as two tile_eval calls.
__device__ __forceinline__ float2 tile_eval2(const float *tile, int p0, int p1, float2 cq, float2 cu, float2 dy,
                                             float2 dx)
{
    const float *a = tile + p0, *b = tile + p1;
    float2 e[4];
    const int off[4] = {0, 1, TS, TS + 1};
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int o = off[i];
        e[i] = __ffma2_rn(cu, make_float2(a[o + 2 * PS], b[o + 2 * PS]),
                          __ffma2_rn(cq, make_float2(a[o + PS], b[o + PS]), make_float2(a[o], b[o])));
    }
    const float2 m1 = make_float2(-1.0f, -1.0f), one = make_float2(1.0f, 1.0f);
    const float2 wy0 = __ffma2_rn(dy, m1, one), wx0 = __ffma2_rn(dx, m1, one);
    float2 r = __fmul2_rn(__fmul2_rn(wy0, wx0), e[0]);
    r = __ffma2_rn(__fmul2_rn(wy0, dx), e[1], r);
    r = __ffma2_rn(__fmul2_rn(dy, wx0), e[2], r);
    return __ffma2_rn(__fmul2_rn(dy, dx), e[3], r);
}

// Response factors of a sample as (ct, cq, cu) = (t_resp, p_resp cos 2a, p_resp sin 2a), or
// (1, cos 2a, sin 2a) without a response.
template<bool RESP>
__device__ __forceinline__ void sample_factors(const OpArgs &a, uint32_t s, float sn, float cs, float &ct, float &cq,
                                               float &cu)
{
    ct = 1.0f;
    cq = cs;
    cu = sn;
    if constexpr (RESP) {
        float tr, pr;
        sample_response(a, s, tr, pr);
        ct = tr;
        cq = pr * cs;
        cu = pr * sn;
    }
}

// One sample of map2tod, general path: exact locate with error bits, then the staged tile or, if the
// footprint is not inside it, global memory.
template<bool RESP, bool PERIODIC>
__device__ __forceinline__ float m2t_sample(const OpArgs &a, const float *tile, const Tile &T, float y, float x,
                                            float al, uint32_t s, uint32_t &err)
{
    Located L;
    err |= locate(y, x, a.ny, a.nx, PERIODIC, L);
    float sn, cs, ct, cq, cu;
    sincos2a(al, &sn, &cs);
    sample_factors<RESP>(a, s, sn, cs, ct, cq, cu);
    int ry, rx;
    if (tile_position<PERIODIC>(L, T, a, ry, rx))
        return tile_eval<RESP>(tile, ry * TS + rx, ct, cq, cu, L.dy, L.dx);
    // Absent cells are already reported through the plan's cell bitmap.
    uint32_t unused = 0;
    const float e00 = global_eval<RESP>(a, a.in, L.iy0, L.ix0, ct, cq, cu, unused);
    const float e01 = global_eval<RESP>(a, a.in, L.iy0, L.ix1, ct, cq, cu, unused);
    const float e10 = global_eval<RESP>(a, a.in, L.iy1, L.ix0, ct, cq, cu, unused);
    const float e11 = global_eval<RESP>(a, a.in, L.iy1, L.ix1, ct, cq, cu, unused);
    return bilinear(L.dy, L.dx, e00, e01, e10, e11);
}

// One sample of tod2map: exact locate with error bits, then shared-memory atomics into the staged
// tile or, if the footprint is not inside it, global atomics.  o0..o2 are this lane's polarisation
// plane offsets in rotated order and 'rot' selects the matching rotation of (t, q, u): in one atomic
// instruction, lanes on the same pixel then target different words.
//
// Flush mode kFlushF32 splits the footprint: its upper row (6 atomics) goes into the tile, its lower
// row (6 reductions) straight into the map at the offsets of the tile's offset table 'tab'.  The
// other flush modes keep every partial in the tile, because their flush is what adds precision.
template<bool RESP, bool PERIODIC, int FLUSH = kFlushF32>
__device__ __forceinline__ void t2m_sample(const OpArgs &a, float *tile, const int64_t *tab, const Tile &T, float y,
                                           float x, float al, float tv, uint32_t s, int rot, int o0, int o1, int o2,
                                           uint32_t &err)
{
    Located L;
    err |= locate(y, x, a.ny, a.nx, PERIODIC, L);
    float sn, cs;
    sincos2a(al, &sn, &cs);
    float t, q, u;
    if constexpr (RESP) {
        float tr, pr;
        sample_response(a, s, tr, pr);
        t = tr * tv;
        q = pr * tv * cs;
        u = pr * tv * sn;
    } else {
        t = tv;
        q = tv * cs;
        u = tv * sn;
    }
    const float wy0 = 1.0f - L.dy, wx0 = 1.0f - L.dx;
    const float w00 = wy0 * wx0, w01 = wy0 * L.dx, w10 = L.dy * wx0, w11 = L.dy * L.dx;
    int ry, rx;
    if (tile_position<PERIODIC>(L, T, a, ry, rx)) {
        const float v0 = (rot == 0) ? t : ((rot == 1) ? q : u);
        const float v1 = (rot == 0) ? q : ((rot == 1) ? u : t);
        const float v2 = (rot == 0) ? u : ((rot == 1) ? t : q);
        const int p = ry * TS + rx;
        float *p0 = tile + p + o0, *p1 = tile + p + o1, *p2 = tile + p + o2;
        atomicAdd(p0, w00 * v0);
        atomicAdd(p1, w00 * v1);
        atomicAdd(p2, w00 * v2);
        atomicAdd(p0 + 1, w01 * v0);
        atomicAdd(p1 + 1, w01 * v1);
        atomicAdd(p2 + 1, w01 * v2);
        if constexpr (FLUSH == kFlushF32) {
            // Lower row: tile row ry + 1 (inside the tile), its two columns' map offsets from 'tab'.
            // An absent cell (offset -1) is skipped, as the flush skips it.
            const int64_t *tb = tab + ((ry + 1) >> 6) * TX + rx;
            const int64_t roff = (int64_t) ((ry + 1) & 63) * a.ystride;
            const int64_t b0 = tb[0], b1 = tb[1];
            const int64_t ps = a.polstride;
            if (b0 >= 0) {
                float *g = a.out + b0 + roff;
                atomicAdd(g, w10 * t);
                atomicAdd(g + ps, w10 * q);
                atomicAdd(g + 2 * ps, w10 * u);
            }
            if (b1 >= 0) {
                float *g = a.out + b1 + roff;
                atomicAdd(g, w11 * t);
                atomicAdd(g + ps, w11 * q);
                atomicAdd(g + 2 * ps, w11 * u);
            }
            return;
        }
        atomicAdd(p0 + TS, w10 * v0);
        atomicAdd(p1 + TS, w10 * v1);
        atomicAdd(p2 + TS, w10 * v2);
        atomicAdd(p0 + TS + 1, w11 * v0);
        atomicAdd(p1 + TS + 1, w11 * v1);
        atomicAdd(p2 + TS + 1, w11 * v2);
    } else {
        uint32_t unused = 0;
        global_accum<FLUSH>(a, a.out, L.iy0, L.ix0, t, q, u, w00, unused);
        global_accum<FLUSH>(a, a.out, L.iy0, L.ix1, t, q, u, w01, unused);
        global_accum<FLUSH>(a, a.out, L.iy1, L.ix0, t, q, u, w10, unused);
        global_accum<FLUSH>(a, a.out, L.iy1, L.ix1, t, q, u, w11, unused);
    }
}

// A sample on the fast path: tile offset, bilinear fractions and sin/cos 2a.
struct TileSample {
    int p;
    float dy, dx, sn, cs;
};

// The common case of locate + tile_position + sincos2a, without branches: true if the sample is
// valid (no error bit), needs no clamp and no x = nx wrap, lies inside the tile and has |2a| <= 1024.
// S then holds what the general path computes from the same operations (bit for bit); otherwise
// S.p = 0 and the caller must take the general path.
template<bool PERIODIC>
__device__ __forceinline__ bool tile_sample(float y, float x, float al, const Tile &T, const OpArgs &a, TileSample &S)
{
    // y in [0, ny-1): trunc(y) is in [0, ny-2], so locate's clamp does nothing.  The truncations of
    // non-negative coordinates go through floor_nonneg (no conversion instructions; the same values).
    bool fast = (y >= 0.0f) && (y < (float) (a.ny - 1));
    float fy;
    const int iy0 = floor_nonneg(y, &fy);
    S.dy = y - fy;
    int ix0;
    float fx;
    if constexpr (PERIODIC) {
        // locate's fold; a folded x in [0, nx) comes only from a valid x and needs no wrap of ix0.
        const float fnx = (float) a.nx;
        float xf = (x >= 0.0f) ? x : (x + fnx);
        xf = (xf <= fnx) ? xf : (xf - fnx);
        fast = fast && (xf >= 0.0f) && (xf < fnx);
        ix0 = floor_nonneg(xf, &fx);
        S.dx = xf - fx;
    } else {
        fast = fast && (x >= 0.0f) && (x < (float) (a.nx - 2));
        ix0 = floor_nonneg(x, &fx);
        S.dx = x - fx;
    }
    const int ry = iy0 - T.gy0;
    int rx = ix0 - T.gx0;
    if constexpr (PERIODIC) {
        rx += (rx < 0) ? a.nx : 0;
        rx -= (rx > TX - 2) ? a.nx : 0;
    }
    fast = fast && ((unsigned) ry <= (unsigned) (TY - 2)) && ((unsigned) rx <= (unsigned) (TX - 2));
    const float th = 2.0f * al;
    fast = fast && (fabsf(th) <= 1024.0f);
    sincos_reduced(th, &S.sn, &S.cs);
    S.p = fast ? (ry * TS + rx) : 0;
    return fast;
}

// Not-in-pixelization check of the plan's cells (this CTA's share of the bitmap; any block size).
__device__ uint32_t check_plan_cells(const uint32_t *__restrict__ cellmap, const OpArgs &a)
{
    uint32_t err = 0;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < kCellmapWords; w += gridDim.x * blockDim.x) {
        uint32_t bits = __ldg(cellmap + w);
        while (bits) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const int c = 32 * w + b;
            const int iy = c >> 10, ix = c & 1023;
            const bool ok = (iy < a.nycells) && (ix < a.nxcells) &&
                            (__ldg(a.cell_offsets + (int64_t) iy * a.nxcells + ix) >= 0);
            err |= ok ? 0u : kErrNotInPixelization;
        }
    }
    return err;
}

// Planned operator kernel.  TOD2MAP selects the direction, RESP the per-detector response and
// PERIODIC the x-wraparound.
//
// A warp takes CH consecutive owner entries at a time; lane i < CH decodes entry i, and two ballots
// give the chunk's usable lines and the first entry of another cell (which ends the CTA's run).
// The lines are then processed UNR at a time with one sample per lane, so the per-line decoding
// costs a shuffle per sample.
template<bool TOD2MAP, bool RESP, bool PERIODIC, int FLUSH = kFlushF32, bool BATCH = false>
__global__ void __launch_bounds__(NT, 2)
planned_kernel(OpArgs a, const uint64_t *__restrict__ owner_mt, int64_t nowner, const uint32_t *__restrict__ cellmap)
{
    static_assert(!BATCH || (TOD2MAP && !RESP), "batched map2tod uses planned_map2tod_v4; no response variant");
    extern __shared__ float tile[];
    __shared__ int s_run[2];
    __shared__ uint32_t s_err[NW];
    __shared__ int64_t s_tab[kTabEntries];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t e0 = (nowner * (int64_t) blockIdx.x) / gridDim.x;
    const int64_t e1 = (nowner * (int64_t) (blockIdx.x + 1)) / gridDim.x;
    const uint32_t nsamp = (uint32_t) a.nsamp;
    const uint32_t nlines = nsamp >> 5;
    const float *__restrict__ yrow = a.xp;
    const float *__restrict__ xrow = a.xp + nsamp;
    const float *__restrict__ arow = a.xp + 2 * (size_t) nsamp;
    uint32_t err = a.partial ? 0u : check_plan_cells(cellmap, a);

    const int rot = lane % 3;
    const int o0 = rot * PS, o1 = ((rot + 1) % 3) * PS, o2 = ((rot + 2) % 3) * PS;

    if constexpr (TOD2MAP) {
        for (int i = threadIdx.x; i < 3 * PS; i += NT)
            tile[i] = 0.0f;
    }

    int64_t start = e0;
    int parity = 0;
    while (start < e1) {
        const uint32_t cell = (uint32_t) (__ldg(owner_mt + start) & kCellMask);
        Tile T;
        T.gy0 = (int) (cell >> 10) << 6;
        T.gx0 = ((int) (cell & 1023u) << 6) - HX;
        // With a run cap (precision modes) a run also ends after max_run_lines entries; the next run
        // then continues the same cell with a fresh tile partial.
        const int64_t erun = ((FLUSH != kFlushF32) && (a.max_run_lines > 0)) ? min(e1, start + a.max_run_lines) : e1;
        if (threadIdx.x == 0)
            s_run[parity] = (int) (erun - start);
        tile_offsets(s_tab, T, a);
        __syncthreads();
        if constexpr (!TOD2MAP) {
            load_tile(tile, s_tab, a, a.in);
            __syncthreads();
        }

        // The next chunk's owner word is fetched while this chunk is processed.
        int64_t c = start + warp * CH;
        uint64_t wnext = ((lane < CH) && (c + lane < erun)) ? __ldg(owner_mt + c + lane) : 0ull;
        for (; c < erun; c += NW * CH) {
            const bool in = (lane < CH) && (c + lane < erun);
            const uint64_t w = wnext;
            const int64_t cn = c + NW * CH;
            wnext = ((lane < CH) && (cn + lane < erun)) ? __ldg(owner_mt + cn + lane) : 0ull;
            // The owner list is sorted by cell: the first entry of another cell ends this run for
            // the whole CTA, and every later entry is past it as well.
            const bool same = in && ((uint32_t) (w & kCellMask) == cell);
            // A plan word always names a line < nsamp/32; anything else means the plan does not
            // belong to this xpointing, so flag it and skip the line.
            const uint32_t line = (uint32_t) ((w >> 20) & kClMask);
            uint32_t nl = nlines;
            if constexpr (BATCH) {
                const uint32_t td = (uint32_t) (w >> kBatchTodShift);
                nl = ((td < (uint32_t) a.ntod) && !(w & kZflag)) ? (uint32_t) (__ldg(&a.descs[td].nsamp) >> 5) : 0u;
            }
            const bool line_ok = line < nl;
            err |= (same && !line_ok) ? kErrInconsistentNmt : 0u;
            const unsigned okmask = __ballot_sync(kFullMask, same && line_ok);
            const unsigned fmask = __ballot_sync(kFullMask, in && !same);
            if ((fmask != 0) && (lane == 0))
                atomicMin(&s_run[parity], (int) (c - start) + __ffs(fmask) - 1);

            for (int g = 0; (g < CH) && ((okmask >> g) != 0u); g += UNR) {
                bool ok[UNR];
                uint32_t s[UNR];
#pragma unroll
                for (int u = 0; u < UNR; u++) {
                    ok[u] = (okmask >> (g + u)) & 1u;
                    s[u] = (__shfl_sync(kFullMask, line, g + u) << 5) + (uint32_t) lane;
                }
                float y[UNR], x[UNR], al[UNR], tv[UNR];
#pragma unroll
                for (int u = 0; u < UNR; u++) {
                    if constexpr (BATCH) {
                        // Rows of the line's TOD (the TOD index is warp-uniform per line).
                        const uint32_t td = __shfl_sync(kFullMask, (uint32_t) (w >> kBatchTodShift), g + u);
                        const gmm_tod_desc *d = a.descs + ((td < (uint32_t) a.ntod) ? td : 0u);
                        const float *yb = (const float *) __ldg((const unsigned long long *) &d->xpointing);
                        const float *tb = (const float *) __ldg((const unsigned long long *) &d->tod);
                        const int64_t ns = __ldg(&d->nsamp);
                        y[u] = ok[u] ? __ldcs(yb + s[u]) : 0.0f;
                        x[u] = ok[u] ? __ldcs(yb + ns + s[u]) : 0.0f;
                        al[u] = ok[u] ? __ldcs(yb + 2 * ns + s[u]) : 0.0f;
                        tv[u] = ok[u] ? __ldcs(tb + s[u]) : 0.0f;
                    } else {
                        y[u] = ok[u] ? __ldcs(yrow + s[u]) : 0.0f;
                        x[u] = ok[u] ? __ldcs(xrow + s[u]) : 0.0f;
                        al[u] = ok[u] ? __ldcs(arow + s[u]) : 0.0f;
                        if constexpr (TOD2MAP)
                            tv[u] = ok[u] ? __ldcs(a.in + s[u]) : 0.0f;
                        else
                            tv[u] = (a.accum && ok[u]) ? a.out[s[u]] : 0.0f;
                    }
                }
#pragma unroll
                for (int u = 0; u < UNR; u++) {
                    if (!ok[u])
                        continue;
                    // tod2map runs the general path for every sample: its time goes to the
                    // atomics, and the vote below would keep the compiler from overlapping one
                    // sample's arithmetic with the previous sample's atomics (measured slower).
                    if constexpr (TOD2MAP) {
                        t2m_sample<RESP, PERIODIC, FLUSH>(a, tile, s_tab, T, y[u], x[u], al[u], tv[u], s[u], rot, o0, o1, o2,
                                                          err);
                    } else {
                        // map2tod: fast path when every lane's sample passes tile_sample (the line
                        // is warp-uniform), else the general path.
                        TileSample S;
                        float r;
                        if (__all_sync(kFullMask, tile_sample<PERIODIC>(y[u], x[u], al[u], T, a, S))) {
                            float ct, cq, cu;
                            sample_factors<RESP>(a, s[u], S.sn, S.cs, ct, cq, cu);
                            r = tile_eval<RESP>(tile, S.p, ct, cq, cu, S.dy, S.dx);
                        } else {
                            r = m2t_sample<RESP, PERIODIC>(a, tile, T, y[u], x[u], al[u], s[u], err);
                        }
                        __stcs(a.out + s[u], a.accum ? (tv[u] + r) : r);
                    }
                }
            }
            if (fmask != 0u)
                break;
        }
        __syncthreads();
        const int64_t next = start + s_run[parity];
        if constexpr (TOD2MAP)
            flush_tile<FLUSH>(tile, s_tab, a, a.out);
        parity ^= 1;
        __syncthreads();
        start = next;
    }
    block_publish_err(err, s_err, a.errword);
}

// map2tod, 16-byte form (xpointing and TOD 16-byte aligned).  A warp takes four owner entries at a
// time: lane group g = lane/8 handles entry g's cache line, each lane four consecutive samples of it,
// so xpointing and TOD move with one float4 load (or store) per lane and row, and the owner word
// needs no shuffle.
template<bool RESP, bool PERIODIC, bool BATCH = false>
__global__ void __launch_bounds__(NT, 2)
planned_map2tod_v4(OpArgs a, const uint64_t *__restrict__ owner_mt, int64_t nowner,
                   const uint32_t *__restrict__ cellmap)
{
    static_assert(!(BATCH && RESP), "batches have no response variant");
    extern __shared__ float tile[];
    __shared__ int s_run[2];
    __shared__ uint32_t s_err[NW];
    __shared__ int64_t s_tab[kTabEntries];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = lane >> 3, sub = lane & 7;
    const int64_t e0 = (nowner * (int64_t) blockIdx.x) / gridDim.x;
    const int64_t e1 = (nowner * (int64_t) (blockIdx.x + 1)) / gridDim.x;
    const uint32_t nsamp = (uint32_t) a.nsamp;
    const uint32_t nlines = nsamp >> 5;
    const float *__restrict__ yrow = a.xp;
    const float *__restrict__ xrow = a.xp + nsamp;
    const float *__restrict__ arow = a.xp + 2 * (size_t) nsamp;
    uint32_t err = a.partial ? 0u : check_plan_cells(cellmap, a);

    int64_t start = e0;
    int parity = 0;
    while (start < e1) {
        const uint32_t cell = (uint32_t) (__ldg(owner_mt + start) & kCellMask);
        Tile T;
        T.gy0 = (int) (cell >> 10) << 6;
        T.gx0 = ((int) (cell & 1023u) << 6) - HX;
        if (threadIdx.x == 0)
            s_run[parity] = (int) (e1 - start);
        tile_offsets(s_tab, T, a);
        __syncthreads();
        load_tile(tile, s_tab, a, a.in);
        __syncthreads();

        int64_t c = start + 4 * warp;
        uint64_t wnext = (c + grp < e1) ? __ldg(owner_mt + c + grp) : 0ull;
        for (; c < e1; c += 4 * NW) {
            const bool in = c + grp < e1;
            const uint64_t w = wnext;
            const int64_t cn = c + 4 * NW;
            wnext = (cn + grp < e1) ? __ldg(owner_mt + cn + grp) : 0ull;
            // The owner list is sorted by cell: the first entry of another cell ends this run.
            const bool same = in && ((uint32_t) (w & kCellMask) == cell);
            const uint32_t line = (uint32_t) ((w >> 20) & kClMask);
            // Rows of this lane's line: the call's arrays, or (batches) those of the line's TOD.
            const float *yb = yrow, *xb = xrow, *ab = arow;
            float *ob = a.out;
            uint32_t nl = nlines;
            if constexpr (BATCH) {
                const uint32_t td = (uint32_t) (w >> kBatchTodShift);
                const gmm_tod_desc *d = a.descs + ((td < (uint32_t) a.ntod) ? td : 0u);
                yb = (const float *) __ldg((const unsigned long long *) &d->xpointing);
                const int64_t ns = __ldg(&d->nsamp);
                xb = yb + ns;
                ab = yb + 2 * ns;
                ob = (float *) __ldg((const unsigned long long *) &d->tod);
                nl = ((td < (uint32_t) a.ntod) && !(w & kZflag)) ? (uint32_t) (ns >> 5) : 0u;
            }
            const bool line_ok = line < nl;
            err |= (same && !line_ok) ? kErrInconsistentNmt : 0u;
            const bool ok = same && line_ok;
            const unsigned fmask = __ballot_sync(kFullMask, in && !same) & 0x01010101u;
            if ((fmask != 0u) && (lane == 0))
                atomicMin(&s_run[parity], (int) (c - start) + ((__ffs(fmask) - 1) >> 3));

            const uint32_t s0 = (line << 5) + 4u * (uint32_t) sub;
            float4 y4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), x4 = y4, a4 = y4, t4 = y4;
            if (ok) {
                y4 = __ldcs(reinterpret_cast<const float4 *>(yb + s0));
                x4 = __ldcs(reinterpret_cast<const float4 *>(xb + s0));
                a4 = __ldcs(reinterpret_cast<const float4 *>(ab + s0));
                if (a.accum)
                    t4 = *reinterpret_cast<const float4 *>(ob + s0);
            }
            const float tv[4] = {t4.x, t4.y, t4.z, t4.w};
            // Fast path when all four samples of every lane pass tile_sample, else the general path.
            TileSample S[4];
            bool fast = tile_sample<PERIODIC>(y4.x, x4.x, a4.x, T, a, S[0]);
            fast = tile_sample<PERIODIC>(y4.y, x4.y, a4.y, T, a, S[1]) && fast;
            fast = tile_sample<PERIODIC>(y4.z, x4.z, a4.z, T, a, S[2]) && fast;
            fast = tile_sample<PERIODIC>(y4.w, x4.w, a4.w, T, a, S[3]) && fast;
            if (__all_sync(kFullMask, fast || !ok)) {
                if (ok) {
                    float r[4];
                    if constexpr (RESP) {
#pragma unroll
                        for (int k = 0; k < 4; k++) {
                            float ct, cq, cu;
                            sample_factors<RESP>(a, s0 + k, S[k].sn, S[k].cs, ct, cq, cu);
                            r[k] = tv[k] + tile_eval<RESP>(tile, S[k].p, ct, cq, cu, S[k].dy, S[k].dx);
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < 4; k += 2) {
                            const float2 e = tile_eval2(tile, S[k].p, S[k + 1].p, make_float2(S[k].cs, S[k + 1].cs),
                                                        make_float2(S[k].sn, S[k + 1].sn), make_float2(S[k].dy, S[k + 1].dy),
                                                        make_float2(S[k].dx, S[k + 1].dx));
                            r[k] = tv[k] + e.x;
                            r[k + 1] = tv[k + 1] + e.y;
                        }
                    }
                    __stcs(reinterpret_cast<float4 *>(ob + s0), make_float4(r[0], r[1], r[2], r[3]));
                }
            } else if (ok) {
                // General path: the pointing is read again rather than kept live across the fast path.
                const float4 yy = __ldcs(reinterpret_cast<const float4 *>(yb + s0));
                const float4 xx = __ldcs(reinterpret_cast<const float4 *>(xb + s0));
                const float4 aa = __ldcs(reinterpret_cast<const float4 *>(ab + s0));
                const float yv[4] = {yy.x, yy.y, yy.z, yy.w};
                const float xv[4] = {xx.x, xx.y, xx.z, xx.w};
                const float av[4] = {aa.x, aa.y, aa.z, aa.w};
                float r[4];
#pragma unroll
                for (int k = 0; k < 4; k++)
                    r[k] = tv[k] + m2t_sample<RESP, PERIODIC>(a, tile, T, yv[k], xv[k], av[k], s0 + k, err);
                __stcs(reinterpret_cast<float4 *>(ob + s0), make_float4(r[0], r[1], r[2], r[3]));
            }
            if (fmask != 0u)
                break;
        }
        __syncthreads();
        const int64_t next = start + s_run[parity];
        parity ^= 1;
        __syncthreads();
        start = next;
    }
    block_publish_err(err, s_err, a.errword);
}

// ------------------------------------------------------------------------------------------------
// Planned tod2map by row bands (single-TOD plans; every flush mode).
//
// The owner list of a single-TOD plan is sorted by (cell, row band, line); the band is the row of a
// line's first sample within its owner cell.  Each warp walks a contiguous range of the list.  While
// the (cell, band) stays the same, it accumulates into a per-warp array in shared memory: rows
// R0 = 64 iycell + band and R0 + 1, columns x0 .. x0 + 95 (x0 = 64 ixcell, unwrapped), planes T, Q,
// U.  A line whose samples all lie in those rows and move by at most one column per sample in one
// direction (a raster scan slower than 1 px/sample, except at its turnarounds; the plan's band word
// says so) is added without atomics: each sample's contribution is split between its two columns,
// the samples of one column are summed by shuffles at the last lane of their run, and those lanes,
// one per column, add their totals into the array with plain read-add-writes in two rounds (own
// column, then the next).  When the (cell, band) changes, or after max_run_lines lines (precision
// modes), the array goes into the map with one L2 reduction per pixel and plane (zeros skipped), in
// flush mode FLUSH; lane L flushes the columns congruent to L mod 32.  Other lines go sample by
// sample straight into the map (twelve reductions each).  Batches use planned_kernel.
//
// Each warp streams its lines through a ring of BP line slots in shared memory (y, x, alpha and TOD
// rows, 512 bytes per line): every lane copies 16 bytes of a line with cp.async, BP - 1 lines ahead
// of the one being processed, so a warp keeps BP - 1 lines of memory traffic in flight while it
// works without holding registers for them.

constexpr int kBandRows = 3;          // accumulator rows R0 .. R0 + 2

// Geometry per flush mode: BW warps per CTA (2 CTAs per SM), BP line slots per warp (a power of
// two).  16 warps with 4 slots (32 warps per SM) measured fastest for the float, float64 and hot-cell
// flushes.  The compensated flush waits on returning atomics at every flush and needs 80 registers:
// at 16 warps (64 registers at most, and shorter warp slices, so more flushes per line) it measured
// 9-11 % slower than with 12 warps and 8 slots.
template<int FLUSH>
struct BandGeo {
    static constexpr int BW = (FLUSH == kFlushCompensated) ? 12 : 16;
    static constexpr int BP = (FLUSH == kFlushCompensated) ? 8 : 4;
    static constexpr int BNT = BW * 32;
    static constexpr size_t kSmem = (size_t) BW * BP * 128 * sizeof(float) + (size_t) BW * 3 * kBandRows * 96 * sizeof(float);
};
constexpr uint32_t kNoKey = 0xffffffffu;

struct BandState {
    float *acc;         // the warp's accumulator in shared memory, rows R0 + [0, 3) (acc_tq, acc_u)
    uint32_t key;       // cell | band << 20 of the accumulated lines, or kNoKey
    bool row2;          // row R0 + 2 may hold non-zero values (a line crossing a row was added)
    int R0, x0;         // rows R0, R0 + 1; columns x0 + [0, 96) (unwrapped; mod nx with PERIODIC)
    float R0f, x0f;     // the same as floats
};

// Accumulator layout, per row r (288 floats): the (T, Q) pairs of the 96 columns, then their U.
__device__ __forceinline__ float2 *acc_tq(float *acc, int r, int c) { return reinterpret_cast<float2 *>(acc + 288 * r) + c; }
__device__ __forceinline__ float *acc_u(float *acc, int r, int c) { return acc + 288 * r + 192 + c; }

// Adds the accumulator into the map (one addition per non-zero pixel and plane, in flush mode FLUSH)
// and clears it.
// Rows and columns outside the map, and absent cells, only ever hold zeros: every line the band path
// takes has its footprint inside the map (absent cells are reported through the plan's cell bitmap).
template<bool PERIODIC, int FLUSH>
__device__ __forceinline__ void band_flush(const OpArgs &a, BandState &B)
{
    const int lane = threadIdx.x & 31;
    if constexpr (FLUSH == kFlushCompensated) {
        // Row by row: the returning atomics of a row's nine values are issued before any two-sum uses
        // one, so that their round trips overlap (one after the other they would cost nine latencies).
#pragma unroll
        for (int r = 0; r < kBandRows; r++) {
            if ((r == 2) && !B.row2)
                break;
            float v[9];
            bool nz = false;
#pragma unroll
            for (int sl = 0; sl < 3; sl++) {
                const float2 tq = *acc_tq(B.acc, r, 32 * sl + lane);
                v[3 * sl] = tq.x;
                v[3 * sl + 1] = tq.y;
                v[3 * sl + 2] = *acc_u(B.acc, r, 32 * sl + lane);
            }
#pragma unroll
            for (int i = 0; i < 9; i++)
                nz = nz || (v[i] != 0.0f);
            if (!__any_sync(kFullMask, nz))
                continue;
            int64_t off[9];
            float old[9];
#pragma unroll
            for (int i = 0; i < 9; i++) {
                const int sl = i / 3, p = i % 3;
                int gx = B.x0 + 32 * sl + lane;
                bool xin = true;
                if constexpr (PERIODIC)
                    gx %= a.nx;
                else
                    xin = gx < a.nx;
                const int64_t o = (xin && (v[i] != 0.0f)) ? global_pixel_offset(B.R0 + r, gx, a) : -1;
                off[i] = (o >= 0) ? (o + p * a.polstride) : -1;
                old[i] = (off[i] >= 0) ? atomicAdd(a.out + off[i], v[i]) : 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 9; i++)
                if (off[i] >= 0)
                    add_rounding_error(a, off[i], old[i], v[i]);
#pragma unroll
            for (int sl = 0; sl < 3; sl++) {
                *acc_tq(B.acc, r, 32 * sl + lane) = make_float2(0.0f, 0.0f);
                *acc_u(B.acc, r, 32 * sl + lane) = 0.0f;
            }
        }
    } else {
#pragma unroll
        for (int sl = 0; sl < 3; sl++) {
            int gx = B.x0 + 32 * sl + lane;
            bool xin = true;
            if constexpr (PERIODIC)
                gx %= a.nx;
            else
                xin = gx < a.nx;
#pragma unroll
            for (int r = 0; r < kBandRows; r++) {
                if ((r == 2) && !B.row2)
                    break;
                float2 *ctq = acc_tq(B.acc, r, 32 * sl + lane);
                float *cu = acc_u(B.acc, r, 32 * sl + lane);
                const float2 tq = *ctq;
                const float t = tq.x, q = tq.y, u = *cu;
                const bool nz = (t != 0.0f) || (q != 0.0f) || (u != 0.0f);
                if (__any_sync(kFullMask, nz) && nz && xin) {
                    if constexpr (FLUSH == kFlushHotF64) {
                        hot_add3(a, B.R0 + r, gx, t, q, u);
                    } else {
                        const int64_t off = global_pixel_offset(B.R0 + r, gx, a);
                        if (off >= 0) {
                            if (t != 0.0f) global_add<FLUSH>(a, off, t);
                            if (q != 0.0f) global_add<FLUSH>(a, off + a.polstride, q);
                            if (u != 0.0f) global_add<FLUSH>(a, off + 2 * a.polstride, u);
                        }
                    }
                }
                *ctq = make_float2(0.0f, 0.0f);
                *cu = 0.0f;
            }
        }
    }
    B.row2 = false;
}

// One cache line (lane = sample) on the band path, whose shape the plan has analysed: 'bw' is its band
// word (gmm_common.cuh), with the fast bit set.  Returns false, having added nothing, if some sample
// has |2a| > 1024 (those go the general way, through sincosf).
template<bool RESP, bool PERIODIC>
__device__ __forceinline__ bool band_line(const OpArgs &a, BandState &B, uint64_t bw, float y, float x,
                                          float al, float tv, uint32_t s)
{
    const int lane = threadIdx.x & 31;
    const float th = 2.0f * al;
    if (!__all_sync(kFullMask, fabsf(th) <= 1024.0f))
        return false;
    const unsigned su = (unsigned) bw;                   // bit i: sample i in the column of sample i - 1
    const bool inc = (bw & kBandInc) != 0ull;
    const bool r3 = (bw & kBandRun3) != 0ull;
    // dy = y - R0 and xr = x - x0 are exact (integers R0 <= y, x0 <= x; the plan checked both).
    const float dy = y - B.R0f;
    float fk;
    const float xr = x - B.x0f;
    const int k = floor_nonneg(xr, &fk);
    const float dx = xr - fk;   // = x - floor(x), exactly

    // Lanes in scan order ("virtual" order): lane order if x increases, reversed if it decreases.
    float sn, cs;
    sincos_reduced(th, &sn, &cs);
    float ft, fq, fu;
    if constexpr (RESP) {
        float tr, pr;
        sample_response(a, s, tr, pr);
        ft = tr * tv;
        fq = pr * tv * cs;
        fu = pr * tv * sn;
    } else {
        ft = tv;
        fq = tv * cs;
        fu = tv * sn;
    }
    const float wy0 = 1.0f - dy;
    const float f[3] = {ft, fq, fu};
    // The previous sample in scan order (lane -+ 1); unused where it does not exist.
    const int src = (lane + (inc ? 31 : 1)) & 31;
    float fp[3];
#pragma unroll
    for (int p = 0; p < 3; p++)
        fp[p] = __shfl_sync(kFullMask, f[p], src);
    const float dyp = __shfl_sync(kFullMask, dy, src);
    const float dxp = __shfl_sync(kFullMask, dx, src);
    // Same column as the previous / next sample in scan order: bits 0 and 1 of su >> lane, swapped
    // for decreasing x.
    const unsigned sl = su >> lane;
    const bool sprev = (inc ? sl : (sl >> 1)) & 1u;
    const bool snext = (inc ? (sl >> 1) : sl) & 1u;
    const bool last = !snext;   // the last sample of its column holds the column's totals
    const float wap = sprev ? 1.0f - dxp : 0.0f, wbp = sprev ? dxp : 0.0f;
    const float wa = 1.0f - dx;
    // The last sample of each column's run adds the column's totals: weights 1 - dx into its column
    // k, dx into k + 1.  Those lanes have distinct k, so two rounds of plain read-add-writes (columns
    // k, then k + 1) never put two lanes on one word.  (k is clamped: a plan used with pointing other
    // than its own gives wrong sums, never an access outside the accumulator.)
    const int kc = (int) min((unsigned) k, 94u);
    // At most two samples per column (no r3): the last one adds the previous one's share too, with
    // the bilinear weights per (row, column) of both samples, in two rounds of read-add-writes at
    // rows 'c' (the accumulator's rows r0, r0 + 1) and columns kc, then kc + 1.  The (T, Q) pair of a
    // pixel moves through the packed float-pair instructions (one fma.rn.f32x2 for two fmaf, the same
    // rounding), as do the row weights.
    auto rounds =[&](float *c, const float *ff, const float *ffp, float ry, float rdy, float ryp, float rdyp) {
        const float2 r01 = make_float2(ry, rdy), p01 = make_float2(ryp, rdyp);
        const float2 A = __fmul2_rn(make_float2(wa, wa), r01), Bq = __fmul2_rn(make_float2(dx, dx), r01);
        const float2 PA = __fmul2_rn(make_float2(wap, wap), p01), PB = __fmul2_rn(make_float2(wbp, wbp), p01);
        const float2 f01 = make_float2(ff[0], ff[1]), fp01 = make_float2(ffp[0], ffp[1]);
        __syncwarp();
        if (last) {
            float2 *t0 = acc_tq(c, 0, kc), *t1 = acc_tq(c, 1, kc);
            float *u0 = acc_u(c, 0, kc), *u1 = acc_u(c, 1, kc);
            const float2 v0 = *t0, v1 = *t1;
            *u0 = fmaf(A.x, ff[2], fmaf(PA.x, ffp[2], *u0));
            *u1 = fmaf(A.y, ff[2], fmaf(PA.y, ffp[2], *u1));
            *t0 = __ffma2_rn(make_float2(A.x, A.x), f01, __ffma2_rn(make_float2(PA.x, PA.x), fp01, v0));
            *t1 = __ffma2_rn(make_float2(A.y, A.y), f01, __ffma2_rn(make_float2(PA.y, PA.y), fp01, v1));
        }
        __syncwarp();
        if (last) {
            float2 *t0 = acc_tq(c, 0, kc + 1), *t1 = acc_tq(c, 1, kc + 1);
            float *u0 = acc_u(c, 0, kc + 1), *u1 = acc_u(c, 1, kc + 1);
            const float2 v0 = *t0, v1 = *t1;
            *u0 = fmaf(Bq.x, ff[2], fmaf(PB.x, ffp[2], *u0));
            *u1 = fmaf(Bq.y, ff[2], fmaf(PB.y, ffp[2], *u1));
            *t0 = __ffma2_rn(make_float2(Bq.x, Bq.x), f01, __ffma2_rn(make_float2(PB.x, PB.x), fp01, v0));
            *t1 = __ffma2_rn(make_float2(Bq.y, Bq.y), f01, __ffma2_rn(make_float2(PB.y, PB.y), fp01, v1));
        }
    };
    if (!r3) {
        if (!(bw & kBandTwoRows)) {
            rounds(B.acc, f, fp, wy0, dy, 1.0f - dyp, dyp);
            return true;
        }
        B.row2 = true;
        // The line crosses a pixel row: samples with upper row R0 + 1 (dy >= 1) go to the
        // accumulator's rows 1, 2 in a second pass, each pass with the other row's samples at zero
        // (the columns' runs are the same in both passes).  dy - 1 is exact for dy in [1, 2).
        const bool row1 = dy >= 1.0f;
        const float dyl = row1 ? dy - 1.0f : dy;
        const float dylp = __shfl_sync(kFullMask, dyl, src);
#pragma unroll
        for (int pass = 0; pass < 2; pass++) {
            float fm[3], fmp[3];
#pragma unroll
            for (int p = 0; p < 3; p++) {
                fm[p] = (row1 == (pass == 1)) ? f[p] : 0.0f;
                fmp[p] = __shfl_sync(kFullMask, fm[p], src);
            }
            rounds(B.acc + 288 * pass, fm, fmp, 1.0f - dyl, dyl, 1.0f - dylp, dylp);
        }
        return true;
    }
    const float V[6] = {wy0 * ft, wy0 * fq, wy0 * fu, dy * ft, dy * fq, dy * fu};
    const float wyp = 1.0f - dyp;
    const float Vp[6] = {wyp * fp[0], wyp * fp[1], wyp * fp[2], dyp * fp[0], dyp * fp[1], dyp * fp[2]};
    // Runs of three or four: pair sums first, then the pair two samples back if it is in the same
    // column (only the last lane of each run uses them, so the others' sums need not be correct).
    float SA[6], SB[6];
#pragma unroll
    for (int p = 0; p < 6; p++) {
        SA[p] = fmaf(wap, Vp[p], wa * V[p]);
        SB[p] = fmaf(wbp, Vp[p], dx * V[p]);
    }
    const int src2 = (lane + (inc ? 30 : 2)) & 31;
    const unsigned sp2 = inc ? (lane > 0 ? (su >> (lane - 1)) : 0u) : ((lane < 30) ? (su >> (lane + 2)) : 0u);
    const bool sprev2 = sprev && (sp2 & 1u);
#pragma unroll
    for (int p = 0; p < 6; p++) {
        const float a2 = __shfl_sync(kFullMask, SA[p], src2);
        const float b2 = __shfl_sync(kFullMask, SB[p], src2);
        SA[p] = sprev2 ? SA[p] + a2 : SA[p];
        SB[p] = sprev2 ? SB[p] + b2 : SB[p];
    }
    __syncwarp();
    if (last) {
        float2 *t0 = acc_tq(B.acc, 0, kc), *t1 = acc_tq(B.acc, 1, kc);
        float2 v0 = *t0, v1 = *t1;
        v0.x += SA[0]; v0.y += SA[1]; v1.x += SA[3]; v1.y += SA[4];
        *acc_u(B.acc, 0, kc) += SA[2];
        *acc_u(B.acc, 1, kc) += SA[5];
        *t0 = v0;
        *t1 = v1;
    }
    __syncwarp();
    if (last) {
        float2 *t0 = acc_tq(B.acc, 0, kc + 1), *t1 = acc_tq(B.acc, 1, kc + 1);
        float2 v0 = *t0, v1 = *t1;
        v0.x += SB[0]; v0.y += SB[1]; v1.x += SB[3]; v1.y += SB[4];
        *acc_u(B.acc, 0, kc + 1) += SB[2];
        *acc_u(B.acc, 1, kc + 1) += SB[5];
        *t0 = v0;
        *t1 = v1;
    }
    return true;
}

// One sample of a line that the band path does not take: exact locate with error bits, then the
// four neighbours straight into the map.
template<bool RESP, bool PERIODIC, int FLUSH>
__device__ __forceinline__ void band_general_sample(const OpArgs &a, float y, float x, float al, float tv, uint32_t s,
                                                    uint32_t &err)
{
    Located L;
    err |= locate(y, x, a.ny, a.nx, PERIODIC, L);
    float sn, cs;
    sincos2a(al, &sn, &cs);
    float t, q, u;
    if constexpr (RESP) {
        float tr, pr;
        sample_response(a, s, tr, pr);
        t = tr * tv;
        q = pr * tv * cs;
        u = pr * tv * sn;
    } else {
        t = tv;
        q = tv * cs;
        u = tv * sn;
    }
    const float wy0 = 1.0f - L.dy, wx0 = 1.0f - L.dx;
    if constexpr (FLUSH == kFlushCompensated) {
        // All twelve returning atomics first, then the two-sums (their round trips overlap).
        const float w[4] = {wy0 * wx0, wy0 * L.dx, L.dy * wx0, L.dy * L.dx};
        const int iy[4] = {L.iy0, L.iy0, L.iy1, L.iy1}, ix[4] = {L.ix0, L.ix1, L.ix0, L.ix1};
        const float f[3] = {t, q, u};
        int64_t off[12];
        float v[12], old[12];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int64_t o = global_pixel_offset(iy[c], ix[c], a);
#pragma unroll
            for (int p = 0; p < 3; p++) {
                off[3 * c + p] = (o >= 0) ? (o + p * a.polstride) : -1;
                v[3 * c + p] = w[c] * f[p];
                old[3 * c + p] = (o >= 0) ? atomicAdd(a.out + off[3 * c + p], v[3 * c + p]) : 0.0f;
            }
        }
#pragma unroll
        for (int i = 0; i < 12; i++)
            if (off[i] >= 0)
                add_rounding_error(a, off[i], old[i], v[i]);
    } else if constexpr (FLUSH == kFlushHotF64) {
        float w = wy0 * wx0;
        hot_add3(a, L.iy0, L.ix0, w * t, w * q, w * u);
        w = wy0 * L.dx;
        hot_add3(a, L.iy0, L.ix1, w * t, w * q, w * u);
        w = L.dy * wx0;
        hot_add3(a, L.iy1, L.ix0, w * t, w * q, w * u);
        w = L.dy * L.dx;
        hot_add3(a, L.iy1, L.ix1, w * t, w * q, w * u);
    } else {
        uint32_t unused = 0;
        global_accum<FLUSH>(a, a.out, L.iy0, L.ix0, t, q, u, wy0 * wx0, unused);
        global_accum<FLUSH>(a, a.out, L.iy0, L.ix1, t, q, u, wy0 * L.dx, unused);
        global_accum<FLUSH>(a, a.out, L.iy1, L.ix0, t, q, u, L.dy * wx0, unused);
        global_accum<FLUSH>(a, a.out, L.iy1, L.ix1, t, q, u, L.dy * L.dx, unused);
    }
}


template<bool RESP, bool PERIODIC, int FLUSH>
__global__ void __launch_bounds__(BandGeo<FLUSH>::BNT, 2)
planned_tod2map_band(OpArgs a, const uint64_t *__restrict__ owner_mt, int64_t nowner,
                     const uint32_t *__restrict__ cellmap, const uint64_t *__restrict__ band)
{
    constexpr int BW = BandGeo<FLUSH>::BW, BP = BandGeo<FLUSH>::BP;
    extern __shared__ __align__(16) float s_lines[];   // [BW][BP][4 rows][32] (y, x, alpha, TOD), then accumulators
    __shared__ uint4 s_wp[BW][64];   // per entry: line, key, band word (low, high)
    __shared__ uint32_t s_err[BW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nw = (int64_t) gridDim.x * BW;
    const int64_t gw = (int64_t) blockIdx.x * BW + warp;
    const int64_t e0 = (nowner * gw) / nw, e1 = (nowner * (gw + 1)) / nw;
    const int64_t n = e1 - e0;
    const uint32_t nsamp = (uint32_t) a.nsamp;
    const uint32_t nlines = nsamp >> 5;
    uint32_t err = a.partial ? 0u : check_plan_cells(cellmap, a);
    float *ring = s_lines + (size_t) warp * BP * 128;
    // This lane's 16-byte piece of every line: row lane/8 (y, x, alpha, TOD), samples 4 (lane%8) + [0, 4).
    const int row = lane >> 3, piece = 4 * (lane & 7);
    const float *__restrict__ src_row = (row < 3) ? (a.xp + (size_t) row * nsamp) : a.in;

    BandState B;
    B.acc = s_lines + (size_t) BW * BP * 128 + (size_t) warp * 3 * kBandRows * 96;
    for (int i = lane; i < 3 * kBandRows * 96; i += 32)
        B.acc[i] = 0.0f;
    __syncwarp();
    B.key = kNoKey;
    B.row2 = false;
    B.R0 = 0;
    B.x0 = 0;
    B.R0f = 0.0f;
    B.x0f = 0.0f;
    int run = 0;   // lines in the accumulator since its last flush (precision modes cap it)
    // The cap of the current run: max_run_lines in the precision modes (only for hot owner cells in
    // the hot-cell mode, whose other cells reduce in float as the plain path does); 0: none.
    const int mrl = (a.max_run_lines < 0x7fffffff) ? (int) a.max_run_lines : 0x7fffffff;
    int cap = (FLUSH == kFlushF32) ? 0 : mrl;
    const int nq = (int) n;   // a warp's range is far below 2^31 entries

    // The warp's decoded owner entries, two groups of 32 in turn: entry q at [q & 63].  Lines >=
    // nlines (a plan that does not belong to this xpointing) are flagged and skipped (0xffffffff).
    uint4 *wp = s_wp[warp];
    // The raw owner and band words of group g (this lane's entry), loaded one group before they are
    // decoded, so that their memory latency is hidden behind a group of lines.
    uint64_t raw_w = 0ull, raw_bw = 0ull;
    auto load_raw = [&](int g) {
        const int q = 32 * g + lane;
        raw_w = (q < nq) ? __ldg(owner_mt + e0 + q) : 0ull;
        raw_bw = (q < nq) ? __ldg(band + e0 + q) : 0ull;
    };
    auto decode = [&](int g) {
        const int q = 32 * g + lane;
        const uint64_t w = raw_w, bw = raw_bw;
        uint32_t line = (q < nq) ? (uint32_t) ((w >> 20) & kClMask) : 0xffffffffu;
        if ((q < nq) && (line >= nlines)) {
            err |= kErrInconsistentNmt;
            line = 0xffffffffu;
        }
        wp[q & 63] = make_uint4(line, (uint32_t) (w & kCellMask) | ((uint32_t) ((w >> kBandShift) & 63u) << 20),
                                (uint32_t) bw, (uint32_t) (bw >> 32));
    };
    load_raw(0);
    decode(0);
    load_raw(1);
    decode(1);
    load_raw(2);
    __syncwarp();

    // Starts the copy of entry q's line into its ring slot (always commits one group, maybe empty).
    auto issue = [&](int q) {
        const uint32_t line = wp[q & 63].x;   // decoded (0xffffffff past the range's end)
        if (line != 0xffffffffu)
            cp_async16(ring + (q & (BP - 1)) * 128 + 32 * row + piece, src_row + (size_t) (32u * line + piece));
        cp_async_commit();
    };

#pragma unroll 1
    for (int q = 0; q < BP - 1; q++)
        issue(q);
#pragma unroll 1
    for (int q0 = 0; q0 < nq; q0 += 32) {
        if (q0 > 0) {
            decode((q0 >> 5) + 1);     // over the group before q0's, which no one reads any more
            load_raw((q0 >> 5) + 2);
        }
        const int qe = min(q0 + 32, nq);
#pragma unroll 1
        for (int q = q0; q < qe; q++) {
            issue(q + BP - 1);         // into the slot of line q - 1, released at the end of that step
            cp_async_wait<BP - 1>();   // this lane's piece of line q has landed
            __syncwarp();
            const uint4 pw = wp[q & 63];
            const uint32_t line = pw.x;
            if (line != 0xffffffffu) {
                const uint32_t key = pw.y;
                const uint64_t bw = (uint64_t) pw.z | ((uint64_t) pw.w << 32);
                const float *slot = ring + (q & (BP - 1)) * 128;
                const float y = slot[lane], x = slot[32 + lane], al = slot[64 + lane], tv = slot[96 + lane];
                const uint32_t s = (line << 5) + (uint32_t) lane;
                if ((key != B.key) || ((cap > 0) && (run >= cap))) {
                    if (B.key != kNoKey)
                        band_flush<PERIODIC, FLUSH>(a, B);
                    B.key = key;
                    B.R0 = ((int) ((key >> 10) & 1023u) << 6) + (int) (key >> 20);
                    B.x0 = (int) (key & 1023u) << 6;
                    B.R0f = (float) B.R0;
                    B.x0f = (float) B.x0;
                    run = 0;
                    if constexpr (FLUSH == kFlushHotF64) {
                        const int iyc = (int) ((key >> 10) & 1023u), ixc = (int) (key & 1023u);
                        const bool hot = (iyc < a.nycells) && (ixc < a.nxcells) &&
                                         (__ldg(a.hot_slot + (int64_t) iyc * a.nxcells + ixc) >= 0);
                        cap = hot ? mrl : 0;
                    }
                }
                if ((bw & kBandFast) && band_line<RESP, PERIODIC>(a, B, bw, y, x, al, tv, s))
                    run++;
                else
                    band_general_sample<RESP, PERIODIC, FLUSH>(a, y, x, al, tv, s, err);
            }
            __syncwarp();              // everyone is done with this slot before it is refilled
        }
    }
    cp_async_wait<0>();
    if (B.key != kNoKey)
        band_flush<PERIODIC, FLUSH>(a, B);
    block_publish_err(err, s_err, a.errword);
}

// ------------------------------------------------------------------------------------------------
// Unplanned operators (map2tod_unplanned.cu:17-71, tod2map_unplanned.cu:17-66): one pass over the
// samples, map accesses straight to global memory.

// Unplanned tod2map by cache lines: one warp per 32 consecutive samples (lane = sample), the next
// line's loads issued before this one is processed.  A line whose samples all lie in one pixel row
// pair (same iy0, ix1 = ix0 + 1) and move by 0 or 1 column per sample in one direction with at most
// four samples per column (a raster scan between 0.25 and 1 px/sample, except at turnarounds) sums
// the samples of each column by one or two shuffle steps, and only the last lane of each column's
// run adds into the map: 12 reductions per column instead of per sample, on distinct addresses.  Other lines add
// sample by sample (map_accumulator, gpu_mm_internals.hpp:299-355).  Error bits as per sample: the
// run's samples touch the pixels its last lane adds to.
template<bool PERIODIC>
__device__ __forceinline__ void unplanned_t2m_line(const OpArgs &a, bool valid, float y, float x, float al, float tv,
                                                   uint32_t &err)
{
    const int lane = threadIdx.x & 31;
    Located L;
    const uint32_t e = locate(y, x, a.ny, a.nx, PERIODIC, L);
    err |= valid ? e : 0u;
    float sn, cs;
    sincos2a(al, &sn, &cs);
    const float t = tv, q = tv * cs, u = tv * sn;
    const int iyA = __shfl_sync(kFullMask, L.iy0, 0);
    const int dk = L.ix0 - __shfl_up_sync(kFullMask, L.ix0, 1);
    const bool ok = valid && (e == 0u) && (L.iy0 == iyA) && (L.ix1 == L.ix0 + 1);
    const unsigned same = __ballot_sync(kFullMask, (lane > 0) && (dk == 0));
    const unsigned up = __ballot_sync(kFullMask, (lane > 0) && (dk == 1));
    const unsigned down = __ballot_sync(kFullMask, (lane > 0) && (dk == -1));
    const unsigned bad = __ballot_sync(kFullMask, !ok);
    const unsigned r3 = same & (same >> 1);   // some column holds three or more samples
    const bool fast = (bad == 0u) && ((same | up | down) == 0xfffffffeu) && ((up == 0u) || (down == 0u)) &&
                      ((r3 & (r3 >> 2)) == 0u);
    if (!fast) {
        if (valid) {
            const float wy0 = 1.0f - L.dy, wx0 = 1.0f - L.dx;
            global_accum(a, a.out, L.iy0, L.ix0, t, q, u, wy0 * wx0, err);
            global_accum(a, a.out, L.iy0, L.ix1, t, q, u, wy0 * L.dx, err);
            global_accum(a, a.out, L.iy1, L.ix0, t, q, u, L.dy * wx0, err);
            global_accum(a, a.out, L.iy1, L.ix1, t, q, u, L.dy * L.dx, err);
        }
        return;
    }
    // Scan order: lane order if x increases, reversed if it decreases.
    const bool inc = down == 0u;
    const float wy0 = 1.0f - L.dy;
    const float V[6] = {wy0 * t, wy0 * q, wy0 * u, L.dy * t, L.dy * q, L.dy * u};
    const int src = (lane + (inc ? 31 : 1)) & 31;
    float Vp[6];
#pragma unroll
    for (int p = 0; p < 6; p++)
        Vp[p] = __shfl_sync(kFullMask, V[p], src);
    const float dxp = __shfl_sync(kFullMask, L.dx, src);
    const unsigned sl = same >> lane;
    const bool sprev = (inc ? sl : (sl >> 1)) & 1u;
    const bool snext = (inc ? (sl >> 1) : sl) & 1u;
    // Column totals over the run so far (weights 1 - dx for this column, dx for the next): this
    // sample and the previous one if it is in the same column; for runs of three or four, plus the
    // pair two samples back.
    const float wap = sprev ? 1.0f - dxp : 0.0f, wbp = sprev ? dxp : 0.0f;
    float SA[6], SB[6];
#pragma unroll
    for (int p = 0; p < 6; p++) {
        SA[p] = fmaf(wap, Vp[p], (1.0f - L.dx) * V[p]);
        SB[p] = fmaf(wbp, Vp[p], L.dx * V[p]);
    }
    if (r3 != 0u) {
        const int src2 = (lane + (inc ? 30 : 2)) & 31;
        const unsigned sp2 = inc ? (lane > 0 ? (same >> (lane - 1)) : 0u) : ((lane < 30) ? (same >> (lane + 2)) : 0u);
        const bool sprev2 = sprev && (sp2 & 1u);
#pragma unroll
        for (int p = 0; p < 6; p++) {
            const float a2 = __shfl_sync(kFullMask, SA[p], src2);
            const float b2 = __shfl_sync(kFullMask, SB[p], src2);
            SA[p] = sprev2 ? SA[p] + a2 : SA[p];
            SB[p] = sprev2 ? SB[p] + b2 : SB[p];
        }
    }
    if (snext)
        return;   // not the last sample of its column: the last one adds this one's share
    int64_t nb[4];
    neighbour_offsets(L, a, nb);
    const int64_t o[4] = {nb[0], nb[2], nb[1], nb[3]};   // (iy0, ix0), (iy1, ix0), (iy0, ix1), (iy1, ix1)
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (o[c] >= 0) {
            const int r = c & 1;     // row of o[c]; columns: own (c < 2) or next
#pragma unroll
            for (int p = 0; p < 3; p++)
                atomicAdd(a.out + o[c] + p * a.polstride, (c < 2) ? SA[3 * r + p] : SB[3 * r + p]);
        } else {
            err |= a.partial ? 0u : kErrNotInPixelization;
        }
    }
}

template<bool PERIODIC>
__global__ void __launch_bounds__(256)
unplanned_tod2map_lines(OpArgs a)
{
    __shared__ uint32_t s_err[8];
    uint32_t err = 0;
    const int lane = threadIdx.x & 31;
    const int64_t nl = (a.nsamp + 31) / 32;
    const int64_t nw = ((int64_t) gridDim.x * blockDim.x) >> 5;
    int64_t l = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    auto load = [&](int64_t line, float &y, float &x, float &al, float &tv) -> bool {
        const int64_t s = 32 * line + lane;
        const bool v = (line < nl) && (s < a.nsamp);
        y = v ? __ldcs(a.xp + s) : 0.0f;
        x = v ? __ldcs(a.xp + a.nsamp + s) : 0.0f;
        al = v ? __ldcs(a.xp + 2 * a.nsamp + s) : 0.0f;
        tv = v ? __ldcs(a.in + s) : 0.0f;
        return v;
    };
    float y, x, al, tv;
    bool v = load(l, y, x, al, tv);
    for (; l < nl; l += nw) {
        float y2, x2, al2, tv2;
        const bool v2 = load(l + nw, y2, x2, al2, tv2);
        unplanned_t2m_line<PERIODIC>(a, v, y, x, al, tv, err);
        y = y2; x = x2; al = al2; tv = tv2; v = v2;
    }
    block_publish_err(err, s_err, a.errword);
}

// Unplanned map2tod: V consecutive samples per thread (16-byte loads and stores when V = 4).
template<int V>
__global__ void __launch_bounds__(256)
unplanned_map2tod_kernel(OpArgs a)
{
    __shared__ uint32_t s_err[8];
    uint32_t err = 0;
    const int64_t nvec = a.nsamp / V;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t v = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; v < nvec; v += stride) {
        const int64_t s0 = v * V;
        float y[V], x[V], al[V], tv[V], r[V];
        if constexpr (V >= 4) {
#pragma unroll
            for (int h = 0; h < V / 4; h++) {
                const int64_t sh = s0 + 4 * h;
                const float4 yy = __ldcs(reinterpret_cast<const float4 *>(a.xp + sh));
                const float4 xx = __ldcs(reinterpret_cast<const float4 *>(a.xp + a.nsamp + sh));
                const float4 aa = __ldcs(reinterpret_cast<const float4 *>(a.xp + 2 * a.nsamp + sh));
                y[4 * h] = yy.x; y[4 * h + 1] = yy.y; y[4 * h + 2] = yy.z; y[4 * h + 3] = yy.w;
                x[4 * h] = xx.x; x[4 * h + 1] = xx.y; x[4 * h + 2] = xx.z; x[4 * h + 3] = xx.w;
                al[4 * h] = aa.x; al[4 * h + 1] = aa.y; al[4 * h + 2] = aa.z; al[4 * h + 3] = aa.w;
                if (a.accum) {
                    const float4 tt = *reinterpret_cast<const float4 *>(a.out + sh);
                    tv[4 * h] = tt.x; tv[4 * h + 1] = tt.y; tv[4 * h + 2] = tt.z; tv[4 * h + 3] = tt.w;
                } else {
                    tv[4 * h] = tv[4 * h + 1] = tv[4 * h + 2] = tv[4 * h + 3] = 0.0f;
                }
            }
        } else {
            y[0] = __ldcs(a.xp + s0);
            x[0] = __ldcs(a.xp + a.nsamp + s0);
            al[0] = __ldcs(a.xp + 2 * a.nsamp + s0);
            tv[0] = a.accum ? a.out[s0] : 0.0f;
        }
#pragma unroll
        for (int k = 0; k < V; k++) {
            Located L;
            err |= locate(y[k], x[k], a.ny, a.nx, a.periodic, L);
            float sn, cs;
            sincos2a(al[k], &sn, &cs);
            int64_t off[4];
            neighbour_offsets(L, a, off);
            const float e00 = eval_at(a, a.in, off[0], cs, sn, err);
            const float e01 = eval_at(a, a.in, off[1], cs, sn, err);
            const float e10 = eval_at(a, a.in, off[2], cs, sn, err);
            const float e11 = eval_at(a, a.in, off[3], cs, sn, err);
            const float rr = bilinear(L.dy, L.dx, e00, e01, e10, e11);
            r[k] = a.accum ? (tv[k] + rr) : rr;
        }
        if constexpr (V >= 4) {
#pragma unroll
            for (int h = 0; h < V / 4; h++)
                __stcs(reinterpret_cast<float4 *>(a.out + s0 + 4 * h),
                       make_float4(r[4 * h], r[4 * h + 1], r[4 * h + 2], r[4 * h + 3]));
        } else {
            __stcs(a.out + s0, r[0]);
        }
    }
    block_publish_err(err, s_err, a.errword);
}

// map2tod uses the 16-byte kernel when xpointing and TOD are 16-byte aligned.  tod2map keeps one
// sample per lane: with four lines in one atomic instruction its shared-memory bank conflicts cost
// more than the wider loads save (measured).

// Grid of the planned kernels: 'ctas_per_sm' CTAs per SM (default 2, all resident), never fewer
// than 'min_lines' cache lines per CTA (default 64) so that small plans reload few tiles.
static int64_t planned_grid(const OpArgs &a, int64_t nowner)
{
    const int64_t per_sm = (a.ctas_per_sm > 0) ? a.ctas_per_sm : 2;
    const int64_t min_lines = (a.min_lines_per_cta > 0) ? a.min_lines_per_cta : 64;
    int64_t g = per_sm * (int64_t) device_sm_count();
    return std::max<int64_t>(1, std::min<int64_t>(g, (nowner + min_lines - 1) / min_lines));
}

template<bool TOD2MAP, bool RESP, bool PERIODIC, int FLUSH = kFlushF32>
cudaError_t launch_planned_impl(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                cudaStream_t stream)
{
    if (nowner <= 0)
        return cudaSuccess;
    const int64_t g = planned_grid(a, nowner);
    if constexpr (!TOD2MAP) {
        if (((((uintptr_t) a.xp) | ((uintptr_t) a.out)) & 15) == 0) {
            static std::atomic<uint64_t> attr_v4_done{0};
            cudaError_t e = set_smem_limit(planned_map2tod_v4<RESP, PERIODIC>, kTileBytes, attr_v4_done);
            if (e != cudaSuccess)
                return e;
            planned_map2tod_v4<RESP, PERIODIC><<<(unsigned) g, NT, kTileBytes, stream>>>(a, owner_mt, nowner, cellmap);
            return cudaGetLastError();
        }
    }
    static std::atomic<uint64_t> attr_done{0};
    cudaError_t e = set_smem_limit(planned_kernel<TOD2MAP, RESP, PERIODIC, FLUSH>, kTileBytes, attr_done);
    if (e != cudaSuccess)
        return e;
    planned_kernel<TOD2MAP, RESP, PERIODIC, FLUSH><<<(unsigned) g, NT, kTileBytes, stream>>>(a, owner_mt, nowner,
                                                                                            cellmap);
    return cudaGetLastError();
}

template<bool TOD2MAP, bool RESP, int FLUSH>
cudaError_t launch_planned_periodic(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                    cudaStream_t stream)
{
    return a.periodic ? launch_planned_impl<TOD2MAP, RESP, true, FLUSH>(a, owner_mt, nowner, cellmap, stream)
                      : launch_planned_impl<TOD2MAP, RESP, false, FLUSH>(a, owner_mt, nowner, cellmap, stream);
}

// Band-path tod2map: one warp per contiguous range of at least 32 owner entries, up to
// ctas_per_sm (default 2) CTAs of BW warps per SM.  Needs xpointing and the TOD 16-byte aligned
// (the cp.async line copies); the caller falls back to the tile kernel otherwise.
template<bool RESP, bool PERIODIC, int FLUSH>
cudaError_t launch_tod2map_band_impl(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner,
                                     const uint32_t *cellmap, const uint64_t *band, cudaStream_t stream)
{
    static std::atomic<uint64_t> attr_done{0};
    using Geo = BandGeo<FLUSH>;
    cudaError_t e = set_smem_limit(planned_tod2map_band<RESP, PERIODIC, FLUSH>, Geo::kSmem, attr_done);
    if (e != cudaSuccess)
        return e;
    const int per_sm = (a.ctas_per_sm > 0) ? a.ctas_per_sm : 2;
    int64_t g = (nowner + 32 * Geo::BW - 1) / (32 * Geo::BW);
    g = std::max<int64_t>(1, std::min<int64_t>(g, (int64_t) per_sm * device_sm_count()));
    planned_tod2map_band<RESP, PERIODIC, FLUSH><<<(unsigned) g, Geo::BNT, Geo::kSmem, stream>>>(a, owner_mt, nowner, cellmap,
                                                                                         band);
    return cudaGetLastError();
}

template<bool RESP, int FLUSH>
cudaError_t launch_tod2map_band(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                const uint64_t *band, cudaStream_t stream)
{
    if (nowner <= 0)
        return cudaSuccess;
    return a.periodic ? launch_tod2map_band_impl<RESP, true, FLUSH>(a, owner_mt, nowner, cellmap, band, stream)
                      : launch_tod2map_band_impl<RESP, false, FLUSH>(a, owner_mt, nowner, cellmap, band, stream);
}

template<bool TOD2MAP, bool RESP>
cudaError_t launch_planned_dispatch(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                    const uint64_t *band, cudaStream_t stream)
{
    if constexpr (TOD2MAP) {
        const bool aligned = ((((uintptr_t) a.xp) | ((uintptr_t) a.in)) & 15) == 0;
        if (a.flush == kFlushHotF64) {
            // Band kernel only, whatever the kernel setting (the C ABI checks the alignment).
            if (!aligned || !band)
                return cudaErrorInvalidValue;
            return launch_tod2map_band<RESP, kFlushHotF64>(a, owner_mt, nowner, cellmap, band, stream);
        }
        if ((g_tod2map_kernel == GMM_TOD2MAP_BANDS) && aligned && band) {
            if (a.flush == kFlushCompensated)
                return launch_tod2map_band<RESP, kFlushCompensated>(a, owner_mt, nowner, cellmap, band, stream);
            if (a.flush == kFlushF64)
                return launch_tod2map_band<RESP, kFlushF64>(a, owner_mt, nowner, cellmap, band, stream);
            return launch_tod2map_band<RESP, kFlushF32>(a, owner_mt, nowner, cellmap, band, stream);
        }
        if (a.flush == kFlushCompensated)
            return launch_planned_periodic<true, RESP, kFlushCompensated>(a, owner_mt, nowner, cellmap, stream);
        if (a.flush == kFlushF64)
            return launch_planned_periodic<true, RESP, kFlushF64>(a, owner_mt, nowner, cellmap, stream);
    }
    return launch_planned_periodic<TOD2MAP, RESP, kFlushF32>(a, owner_mt, nowner, cellmap, stream);
}

__global__ void fold_compensation_kernel(float *__restrict__ lmap, float *__restrict__ comp, int64_t n)
{
    for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const float c = comp[i];
        if (c != 0.0f) {
            lmap[i] += c;
            comp[i] = 0.0f;
        }
    }
}

template<bool TOD2MAP>
cudaError_t launch_unplanned_impl(const OpArgs &a, cudaStream_t stream)
{
    if constexpr (TOD2MAP) {
        int64_t g = 8 * (int64_t) device_sm_count();
        g = std::max<int64_t>(1, std::min<int64_t>(g, (a.nsamp + 255) / 256));
        if (a.periodic)
            unplanned_tod2map_lines<true><<<(unsigned) g, 256, 0, stream>>>(a);
        else
            unplanned_tod2map_lines<false><<<(unsigned) g, 256, 0, stream>>>(a);
    } else {
        const bool aligned = ((((uintptr_t) a.xp) | ((uintptr_t) a.out)) & 15) == 0;
        const bool vec = aligned && ((a.nsamp & 3) == 0);
        const int64_t nvec = vec ? a.nsamp / 4 : a.nsamp;
        int64_t g = 8 * (int64_t) device_sm_count();
        g = std::max<int64_t>(1, std::min<int64_t>(g, (nvec + 255) / 256));
        if (vec)
            unplanned_map2tod_kernel<4><<<(unsigned) g, 256, 0, stream>>>(a);
        else
            unplanned_map2tod_kernel<1><<<(unsigned) g, 256, 0, stream>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_planned_map2tod(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   cudaStream_t stream)
{
    return a.response ? launch_planned_dispatch<false, true>(a, owner_mt, nowner, cellmap, nullptr, stream)
                      : launch_planned_dispatch<false, false>(a, owner_mt, nowner, cellmap, nullptr, stream);
}

cudaError_t launch_planned_tod2map(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   const uint64_t *band, cudaStream_t stream)
{
    return a.response ? launch_planned_dispatch<true, true>(a, owner_mt, nowner, cellmap, band, stream)
                      : launch_planned_dispatch<true, false>(a, owner_mt, nowner, cellmap, band, stream);
}

template<bool PERIODIC>
cudaError_t launch_batch_map2tod_impl(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner,
                                      const uint32_t *cellmap, cudaStream_t stream)
{
    static std::atomic<uint64_t> attr_done{0};
    cudaError_t e = set_smem_limit(planned_map2tod_v4<false, PERIODIC, true>, kTileBytes, attr_done);
    if (e != cudaSuccess)
        return e;
    planned_map2tod_v4<false, PERIODIC, true><<<(unsigned) planned_grid(a, nowner), NT, kTileBytes, stream>>>(
        a, owner_mt, nowner, cellmap);
    return cudaGetLastError();
}

template<bool PERIODIC>
cudaError_t launch_batch_tod2map_impl(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner,
                                      const uint32_t *cellmap, cudaStream_t stream)
{
    static std::atomic<uint64_t> attr_done{0};
    cudaError_t e = set_smem_limit(planned_kernel<true, false, PERIODIC, kFlushF32, true>, kTileBytes, attr_done);
    if (e != cudaSuccess)
        return e;
    planned_kernel<true, false, PERIODIC, kFlushF32, true><<<(unsigned) planned_grid(a, nowner), NT, kTileBytes, stream>>>(
        a, owner_mt, nowner, cellmap);
    return cudaGetLastError();
}

cudaError_t launch_fold_compensation(float *lmap, float *comp, int64_t n, cudaStream_t stream)
{
    if (n <= 0)
        return cudaSuccess;
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8 * (int64_t) device_sm_count()));
    fold_compensation_kernel<<<(unsigned) g, 256, 0, stream>>>(lmap, comp, n);
    return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------------
// Hot cells: the cells whose partial sums tod2map reduces in float64 (flush mode kFlushHotF64).
//
// plan_cell_lines_kernel adds, for every cell of the local pixelization's grid, the number of plan
// mt words (= cache lines touching the cell) into lines[iycell * nxcells + ixcell].  The words are
// sorted by cell, so the lanes of a warp mostly share one cell: one atomic per distinct cell.

__global__ void plan_cell_lines_kernel(const uint64_t *__restrict__ mt, int64_t nmt, int nycells, int nxcells,
                                       uint32_t *__restrict__ lines)
{
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t i0 = (int64_t) blockIdx.x * blockDim.x; i0 < nmt; i0 += stride) {
        const int64_t i = i0 + threadIdx.x;
        int c = -1;
        if (i < nmt) {
            const uint64_t w = __ldg(mt + i);
            const int ixc = (int) (w & 1023u), iyc = (int) ((w >> 10) & 1023u);
            c = ((iyc < nycells) && (ixc < nxcells)) ? iyc * nxcells + ixc : -1;
        }
        const unsigned peers = __match_any_sync(kFullMask, c);
        if ((c >= 0) && ((peers & ((1u << lane) - 1u)) == 0u))
            atomicAdd(lines + c, (uint32_t) __popc(peers));
    }
}

// One CTA of 1024 threads: slot[c] = rank of cell c among the present cells with lines[c] >=
// min_lines (in cell order), else -1; cells[slot] = c; *nhot = the number of hot cells.
__global__ void __launch_bounds__(1024) hot_cells_kernel(const uint32_t *__restrict__ lines,
                                                         const int64_t *__restrict__ cell_offsets, int ncells,
                                                         uint32_t min_lines, int32_t *__restrict__ slot,
                                                         int32_t *__restrict__ cells, int32_t *__restrict__ nhot)
{
    __shared__ int s_warp[32];
    __shared__ int s_base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0)
        s_base = 0;
    __syncthreads();
    for (int c0 = 0; c0 < ncells; c0 += 1024) {
        const int c = c0 + threadIdx.x;
        const bool hot = (c < ncells) && (lines[c] >= min_lines) && (cell_offsets[c] >= 0);
        const unsigned b = __ballot_sync(kFullMask, hot);
        if (lane == 0)
            s_warp[warp] = __popc(b);
        __syncthreads();
        if (warp == 0) {
            const int v = s_warp[lane];
            int incl = v;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int u = __shfl_up_sync(kFullMask, incl, d);
                incl += (lane >= d) ? u : 0;
            }
            s_warp[lane] = incl - v;   // exclusive prefix over warps
        }
        __syncthreads();
        const int r = s_base + s_warp[warp] + __popc(b & ((1u << lane) - 1u));
        if (c < ncells) {
            slot[c] = hot ? r : -1;
            if (hot)
                cells[r] = c;
        }
        __syncthreads();
        if (threadIdx.x == 1023)
            s_base = r + (hot ? 1 : 0);
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *nhot = s_base;
}

// One CTA per hot cell: local_map = float(local_map + hot) at every non-zero accumulator value (one
// rounding), then the accumulator is zeroed.
__global__ void fold_hot_kernel(float *__restrict__ lmap, double *__restrict__ hot, const int32_t *__restrict__ cells,
                                const int64_t *__restrict__ cell_offsets, int64_t ystride, int64_t polstride)
{
    const int64_t base = cell_offsets[cells[blockIdx.x]];
    if (base < 0)      // the cell left the pixelization after the hot cells were chosen
        return;
    double *h = hot + (int64_t) blockIdx.x * kHotCellDoubles;
    for (int i = threadIdx.x; i < (int) kHotCellDoubles; i += blockDim.x) {
        const double v = h[i];
        if (v != 0.0) {
            const int p = i >> 12, iy = (i >> 6) & 63, ix = i & 63;
            float *m = lmap + base + p * polstride + iy * ystride + ix;
            *m = (float) ((double) *m + v);
            h[i] = 0.0;
        }
    }
}

cudaError_t launch_plan_cell_lines(const uint64_t *mt, int64_t nmt, int nycells, int nxcells, uint32_t *lines,
                                   cudaStream_t stream)
{
    if (nmt <= 0)
        return cudaSuccess;
    const int64_t g = std::max<int64_t>(1, std::min<int64_t>((nmt + 255) / 256, 8 * (int64_t) device_sm_count()));
    plan_cell_lines_kernel<<<(unsigned) g, 256, 0, stream>>>(mt, nmt, nycells, nxcells, lines);
    return cudaGetLastError();
}

cudaError_t launch_hot_cells(const uint32_t *lines, const int64_t *cell_offsets, int ncells, uint32_t min_lines,
                             int32_t *slot, int32_t *cells, int32_t *nhot, cudaStream_t stream)
{
    hot_cells_kernel<<<1, 1024, 0, stream>>>(lines, cell_offsets, ncells, min_lines, slot, cells, nhot);
    return cudaGetLastError();
}

cudaError_t launch_fold_hot(float *lmap, double *hot, const int32_t *cells, int64_t nhot, const int64_t *cell_offsets,
                            int64_t ystride, int64_t polstride, cudaStream_t stream)
{
    if (nhot <= 0)
        return cudaSuccess;
    fold_hot_kernel<<<(unsigned) nhot, 512, 0, stream>>>(lmap, hot, cells, cell_offsets, ystride, polstride);
    return cudaGetLastError();
}

cudaError_t launch_batch_map2tod(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                 cudaStream_t stream)
{
    if (nowner <= 0)
        return cudaSuccess;
    return a.periodic ? launch_batch_map2tod_impl<true>(a, owner_mt, nowner, cellmap, stream)
                      : launch_batch_map2tod_impl<false>(a, owner_mt, nowner, cellmap, stream);
}

cudaError_t launch_batch_tod2map(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                 cudaStream_t stream)
{
    if (nowner <= 0)
        return cudaSuccess;
    return a.periodic ? launch_batch_tod2map_impl<true>(a, owner_mt, nowner, cellmap, stream)
                      : launch_batch_tod2map_impl<false>(a, owner_mt, nowner, cellmap, stream);
}

cudaError_t launch_unplanned_map2tod(const OpArgs &a, cudaStream_t stream)
{
    return launch_unplanned_impl<false>(a, stream);
}

cudaError_t launch_unplanned_tod2map(const OpArgs &a, cudaStream_t stream)
{
    return launch_unplanned_impl<true>(a, stream);
}

}  // namespace gmm
