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
//  * xpointing and TOD are streamed with evict-first loads/stores so that the map and plan stay in
//    L2; each warp keeps UNR cache lines in flight.
#include <algorithm>

#include "gmm_internal.hpp"

namespace gmm {

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

__device__ __forceinline__ int64_t tile_pixel_offset(int r, int c, const Tile &T, const OpArgs &a)
{
    const int gy = T.gy0 + r;
    int gx = T.gx0 + c;
    if (a.periodic) {
        gx %= a.nx;
        gx += (gx < 0) ? a.nx : 0;
    }
    if ((gx < 0) || (gy >= 64 * a.nycells) || (gx >= 64 * a.nxcells))
        return -1;
    const int64_t off = __ldg(a.cell_offsets + (int64_t) (gy >> 6) * a.nxcells + (gx >> 6));
    if (off < 0)
        return -1;
    return off + (int64_t) (gy & 63) * a.ystride + (gx & 63);
}

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

// Loads the tile of 'cell' from the local map (absent pixels read as zero).
__device__ void load_tile(float *tile, const Tile &T, const OpArgs &a, const float *__restrict__ lmap)
{
    for (int idx = threadIdx.x; idx < TY * TX; idx += NT) {
        const int r = idx / TX, c = idx % TX;
        const int64_t off = tile_pixel_offset(r, c, T, a);
        const bool p = off >= 0;
        float *dst = tile + r * TS + c;
        dst[0] = p ? __ldg(lmap + off) : 0.0f;
        dst[PS] = p ? __ldg(lmap + off + a.polstride) : 0.0f;
        dst[2 * PS] = p ? __ldg(lmap + off + 2 * a.polstride) : 0.0f;
    }
}

// Adds the tile into the map (one atomic per non-zero pixel and polarisation) and clears it.
__device__ void flush_tile(float *tile, const Tile &T, const OpArgs &a, float *__restrict__ lmap)
{
    for (int idx = threadIdx.x; idx < TY * TX; idx += NT) {
        const int r = idx / TX, c = idx % TX;
        float *src = tile + r * TS + c;
        const float t = src[0], q = src[PS], u = src[2 * PS];
        if ((t != 0.0f) || (q != 0.0f) || (u != 0.0f)) {
            const int64_t off = tile_pixel_offset(r, c, T, a);
            if (off >= 0) {
                atomicAdd(lmap + off, t);
                atomicAdd(lmap + off + a.polstride, q);
                atomicAdd(lmap + off + 2 * a.polstride, u);
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

__device__ __forceinline__ float global_eval(const OpArgs &a, const float *__restrict__ lmap, int iy, int ix,
                                             float ct, float cq, float cu, uint32_t &err)
{
    const int64_t off = global_pixel_offset(iy, ix, a);
    const bool valid = off >= 0;
    const float t = valid ? __ldg(lmap + off) : 0.0f;
    const float q = valid ? __ldg(lmap + off + a.polstride) : 0.0f;
    const float u = valid ? __ldg(lmap + off + 2 * a.polstride) : 0.0f;
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
    return ct * t + cq * q + cu * u;
}

__device__ __forceinline__ void global_accum(const OpArgs &a, float *__restrict__ lmap, int iy, int ix,
                                             float t, float q, float u, float w, uint32_t &err)
{
    const int64_t off = global_pixel_offset(iy, ix, a);
    const bool valid = off >= 0;
    if (valid) {
        atomicAdd(lmap + off, w * t);
        atomicAdd(lmap + off + a.polstride, w * q);
        atomicAdd(lmap + off + 2 * a.polstride, w * u);
    }
    err |= (valid || a.partial) ? 0u : kErrNotInPixelization;
}

// One sample of map2tod against the staged tile (or global memory if it does not fit).
template<bool RESP, bool PERIODIC>
__device__ __forceinline__ float m2t_sample(const OpArgs &a, const float *tile, const Tile &T, float y, float x,
                                            float al, uint32_t s, uint32_t &err)
{
    Located L;
    err |= locate(y, x, a.ny, a.nx, PERIODIC, L);
    float sn, cs;
    sincos2a(al, &sn, &cs);
    float ct = 1.0f, cq = cs, cu = sn;
    if constexpr (RESP) {
        float tr, pr;
        sample_response(a, s, tr, pr);
        ct = tr;
        cq = pr * cs;
        cu = pr * sn;
    }
    int ry, rx;
    float e00, e01, e10, e11;
    if (tile_position<PERIODIC>(L, T, a, ry, rx)) {
        const float *p = tile + ry * TS + rx;
        if constexpr (RESP) {
            e00 = ct * p[0] + cq * p[PS] + cu * p[2 * PS];
            e01 = ct * p[1] + cq * p[PS + 1] + cu * p[2 * PS + 1];
            e10 = ct * p[TS] + cq * p[PS + TS] + cu * p[2 * PS + TS];
            e11 = ct * p[TS + 1] + cq * p[PS + TS + 1] + cu * p[2 * PS + TS + 1];
        } else {
            e00 = p[0] + cq * p[PS] + cu * p[2 * PS];
            e01 = p[1] + cq * p[PS + 1] + cu * p[2 * PS + 1];
            e10 = p[TS] + cq * p[PS + TS] + cu * p[2 * PS + TS];
            e11 = p[TS + 1] + cq * p[PS + TS + 1] + cu * p[2 * PS + TS + 1];
        }
    } else {
        // Absent cells are already reported through the plan's cell bitmap.
        uint32_t unused = 0;
        e00 = global_eval(a, a.in, L.iy0, L.ix0, ct, cq, cu, unused);
        e01 = global_eval(a, a.in, L.iy0, L.ix1, ct, cq, cu, unused);
        e10 = global_eval(a, a.in, L.iy1, L.ix0, ct, cq, cu, unused);
        e11 = global_eval(a, a.in, L.iy1, L.ix1, ct, cq, cu, unused);
    }
    const float wy0 = 1.0f - L.dy, wx0 = 1.0f - L.dx;
    float r = (wy0 * wx0) * e00;
    r += (wy0 * L.dx) * e01;
    r += (L.dy * wx0) * e10;
    r += (L.dy * L.dx) * e11;
    return r;
}

// One sample of tod2map.  o0..o2 are this lane's polarisation plane offsets in rotated order and
// 'rot' selects the matching rotation of (t, q, u).
template<bool RESP, bool PERIODIC>
__device__ __forceinline__ void t2m_sample(const OpArgs &a, float *tile, const Tile &T, float y, float x, float al,
                                           float tv, uint32_t s, int rot, int o0, int o1, int o2, uint32_t &err)
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
        atomicAdd(p0 + TS, w10 * v0);
        atomicAdd(p1 + TS, w10 * v1);
        atomicAdd(p2 + TS, w10 * v2);
        atomicAdd(p0 + TS + 1, w11 * v0);
        atomicAdd(p1 + TS + 1, w11 * v1);
        atomicAdd(p2 + TS + 1, w11 * v2);
    } else {
        uint32_t unused = 0;
        global_accum(a, a.out, L.iy0, L.ix0, t, q, u, w00, unused);
        global_accum(a, a.out, L.iy0, L.ix1, t, q, u, w01, unused);
        global_accum(a, a.out, L.iy1, L.ix0, t, q, u, w10, unused);
        global_accum(a, a.out, L.iy1, L.ix1, t, q, u, w11, unused);
    }
}

// Not-in-pixelization check of the plan's cells (this CTA's share of the bitmap).
__device__ uint32_t check_plan_cells(const uint32_t *__restrict__ cellmap, const OpArgs &a)
{
    uint32_t err = 0;
    for (int w = blockIdx.x * NT + threadIdx.x; w < kCellmapWords; w += gridDim.x * NT) {
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
template<bool TOD2MAP, bool RESP, bool PERIODIC>
__global__ void __launch_bounds__(NT, 2)
planned_kernel(OpArgs a, const uint64_t *__restrict__ owner_mt, int64_t nowner, const uint32_t *__restrict__ cellmap)
{
    extern __shared__ float tile[];
    __shared__ int s_run[2];
    __shared__ uint32_t s_err[NW];

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
        if (threadIdx.x == 0)
            s_run[parity] = (int) (e1 - start);
        if constexpr (!TOD2MAP)
            load_tile(tile, T, a, a.in);
        __syncthreads();

        // The next chunk's owner word is fetched while this chunk is processed.
        int64_t c = start + warp * CH;
        uint64_t wnext = ((lane < CH) && (c + lane < e1)) ? __ldg(owner_mt + c + lane) : 0ull;
        for (; c < e1; c += NW * CH) {
            const bool in = (lane < CH) && (c + lane < e1);
            const uint64_t w = wnext;
            const int64_t cn = c + NW * CH;
            wnext = ((lane < CH) && (cn + lane < e1)) ? __ldg(owner_mt + cn + lane) : 0ull;
            // The owner list is sorted by cell: the first entry of another cell ends this run for
            // the whole CTA, and every later entry is past it as well.
            const bool same = in && ((uint32_t) (w & kCellMask) == cell);
            // A plan word always names a line < nsamp/32; anything else means the plan does not
            // belong to this xpointing, so flag it and skip the line.
            const uint32_t line = (uint32_t) ((w >> 20) & kClMask);
            const bool line_ok = line < nlines;
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
                    y[u] = ok[u] ? __ldcs(yrow + s[u]) : 0.0f;
                    x[u] = ok[u] ? __ldcs(xrow + s[u]) : 0.0f;
                    al[u] = ok[u] ? __ldcs(arow + s[u]) : 0.0f;
                    if constexpr (TOD2MAP)
                        tv[u] = ok[u] ? __ldcs(a.in + s[u]) : 0.0f;
                    else
                        tv[u] = (a.accum && ok[u]) ? a.out[s[u]] : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < UNR; u++) {
                    if (!ok[u])
                        continue;
                    if constexpr (TOD2MAP) {
                        t2m_sample<RESP, PERIODIC>(a, tile, T, y[u], x[u], al[u], tv[u], s[u], rot, o0, o1, o2, err);
                    } else {
                        const float r = m2t_sample<RESP, PERIODIC>(a, tile, T, y[u], x[u], al[u], s[u], err);
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
            flush_tile(tile, T, a, a.out);
        parity ^= 1;
        __syncthreads();
        start = next;
    }
    block_publish_err(err, s_err, a.errword);
}

// Planned operator kernel, 16-byte form (xpointing and TOD 16-byte aligned).  A warp takes four
// owner entries at a time: lane group g = lane/8 handles entry g's cache line, each lane four
// consecutive samples of it, so xpointing and TOD move with one float4 load (or store) per lane
// and row, and the owner word needs no shuffle.
template<bool TOD2MAP, bool RESP, bool PERIODIC>
__global__ void __launch_bounds__(NT, 2)
planned_kernel_v4(OpArgs a, const uint64_t *__restrict__ owner_mt, int64_t nowner,
                  const uint32_t *__restrict__ cellmap)
{
    extern __shared__ float tile[];
    __shared__ int s_run[2];
    __shared__ uint32_t s_err[NW];

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
        if (threadIdx.x == 0)
            s_run[parity] = (int) (e1 - start);
        if constexpr (!TOD2MAP)
            load_tile(tile, T, a, a.in);
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
            const bool line_ok = line < nlines;
            err |= (same && !line_ok) ? kErrInconsistentNmt : 0u;
            const bool ok = same && line_ok;
            const unsigned fmask = __ballot_sync(kFullMask, in && !same) & 0x01010101u;
            if ((fmask != 0u) && (lane == 0))
                atomicMin(&s_run[parity], (int) (c - start) + ((__ffs(fmask) - 1) >> 3));

            if (ok) {
                const uint32_t s0 = (line << 5) + 4u * (uint32_t) sub;
                const float4 y4 = __ldcs(reinterpret_cast<const float4 *>(yrow + s0));
                const float4 x4 = __ldcs(reinterpret_cast<const float4 *>(xrow + s0));
                const float4 a4 = __ldcs(reinterpret_cast<const float4 *>(arow + s0));
                float4 t4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if constexpr (TOD2MAP)
                    t4 = __ldcs(reinterpret_cast<const float4 *>(a.in + s0));
                else if (a.accum)
                    t4 = *reinterpret_cast<const float4 *>(a.out + s0);
                const float yv[4] = {y4.x, y4.y, y4.z, y4.w};
                const float xv[4] = {x4.x, x4.y, x4.z, x4.w};
                const float av[4] = {a4.x, a4.y, a4.z, a4.w};
                const float tv[4] = {t4.x, t4.y, t4.z, t4.w};
                if constexpr (TOD2MAP) {
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        t2m_sample<RESP, PERIODIC>(a, tile, T, yv[k], xv[k], av[k], tv[k], s0 + k, rot, o0, o1, o2,
                                                   err);
                } else {
                    float r[4];
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        r[k] = tv[k] + m2t_sample<RESP, PERIODIC>(a, tile, T, yv[k], xv[k], av[k], s0 + k, err);
                    __stcs(reinterpret_cast<float4 *>(a.out + s0), make_float4(r[0], r[1], r[2], r[3]));
                }
            }
            if (fmask != 0u)
                break;
        }
        __syncthreads();
        const int64_t next = start + s_run[parity];
        if constexpr (TOD2MAP)
            flush_tile(tile, T, a, a.out);
        parity ^= 1;
        __syncthreads();
        start = next;
    }
    block_publish_err(err, s_err, a.errword);
}

// ------------------------------------------------------------------------------------------------
// Unplanned operators (map2tod_unplanned.cu:17-71, tod2map_unplanned.cu:17-66): one pass over the
// samples, map accesses straight to global memory.  Four consecutive samples per thread with
// 16-byte loads when the arrays are aligned.

template<bool TOD2MAP, int V>
__global__ void __launch_bounds__(256)
unplanned_kernel(OpArgs a)
{
    __shared__ uint32_t s_err[8];
    uint32_t err = 0;
    const int64_t nvec = a.nsamp / V;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x;
    for (int64_t v = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; v < nvec; v += stride) {
        const int64_t s0 = v * V;
        float y[V], x[V], al[V], tv[V], r[V];
        if constexpr (V == 4) {
            const float4 yy = __ldcs(reinterpret_cast<const float4 *>(a.xp + s0));
            const float4 xx = __ldcs(reinterpret_cast<const float4 *>(a.xp + a.nsamp + s0));
            const float4 aa = __ldcs(reinterpret_cast<const float4 *>(a.xp + 2 * a.nsamp + s0));
            y[0] = yy.x; y[1] = yy.y; y[2] = yy.z; y[3] = yy.w;
            x[0] = xx.x; x[1] = xx.y; x[2] = xx.z; x[3] = xx.w;
            al[0] = aa.x; al[1] = aa.y; al[2] = aa.z; al[3] = aa.w;
            if (TOD2MAP || a.accum) {
                const float4 tt = TOD2MAP ? __ldcs(reinterpret_cast<const float4 *>(a.in + s0))
                                          : *reinterpret_cast<const float4 *>(a.out + s0);
                tv[0] = tt.x; tv[1] = tt.y; tv[2] = tt.z; tv[3] = tt.w;
            } else {
                tv[0] = tv[1] = tv[2] = tv[3] = 0.0f;
            }
        } else {
            y[0] = __ldcs(a.xp + s0);
            x[0] = __ldcs(a.xp + a.nsamp + s0);
            al[0] = __ldcs(a.xp + 2 * a.nsamp + s0);
            tv[0] = TOD2MAP ? __ldcs(a.in + s0) : (a.accum ? a.out[s0] : 0.0f);
        }
#pragma unroll
        for (int k = 0; k < V; k++) {
            Located L;
            err |= locate(y[k], x[k], a.ny, a.nx, a.periodic, L);
            float sn, cs;
            sincos2a(al[k], &sn, &cs);
            const float wy0 = 1.0f - L.dy, wx0 = 1.0f - L.dx;
            if constexpr (TOD2MAP) {
                const float t = tv[k], q = t * cs, u = t * sn;
                global_accum(a, a.out, L.iy0, L.ix0, t, q, u, wy0 * wx0, err);
                global_accum(a, a.out, L.iy0, L.ix1, t, q, u, wy0 * L.dx, err);
                global_accum(a, a.out, L.iy1, L.ix0, t, q, u, L.dy * wx0, err);
                global_accum(a, a.out, L.iy1, L.ix1, t, q, u, L.dy * L.dx, err);
            } else {
                float rr = (wy0 * wx0) * global_eval(a, a.in, L.iy0, L.ix0, 1.0f, cs, sn, err);
                rr += (wy0 * L.dx) * global_eval(a, a.in, L.iy0, L.ix1, 1.0f, cs, sn, err);
                rr += (L.dy * wx0) * global_eval(a, a.in, L.iy1, L.ix0, 1.0f, cs, sn, err);
                rr += (L.dy * L.dx) * global_eval(a, a.in, L.iy1, L.ix1, 1.0f, cs, sn, err);
                r[k] = a.accum ? (tv[k] + rr) : rr;
            }
        }
        if constexpr (!TOD2MAP) {
            if constexpr (V == 4)
                __stcs(reinterpret_cast<float4 *>(a.out + s0), make_float4(r[0], r[1], r[2], r[3]));
            else
                __stcs(a.out + s0, r[0]);
        }
    }
    block_publish_err(err, s_err, a.errword);
}

// Which directions use the 16-byte kernel when the arrays allow it.  tod2map keeps one sample per
// lane: with four lines in one atomic instruction its shared-memory bank conflicts cost more than
// the wider loads save.
constexpr bool kVecMap2tod = true;
constexpr bool kVecTod2map = false;   // its atomics conflict more in shared-memory banks

template<bool TOD2MAP, bool RESP, bool PERIODIC>
cudaError_t launch_planned_impl(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                cudaStream_t stream)
{
    if (nowner <= 0)
        return cudaSuccess;
    // Two CTAs per SM; never fewer than ~64 cache lines per CTA, so small plans reload few tiles.
    int64_t g = 2 * (int64_t) device_sm_count();
    g = std::max<int64_t>(1, std::min<int64_t>(g, (nowner + 63) / 64));
    if constexpr (TOD2MAP ? kVecTod2map : kVecMap2tod) {
        const float *tod = TOD2MAP ? a.in : a.out;
        if (((((uintptr_t) a.xp) | ((uintptr_t) tod)) & 15) == 0) {
            static std::atomic<uint64_t> attr_v4_done{0};
            cudaError_t e = set_smem_limit(planned_kernel_v4<TOD2MAP, RESP, PERIODIC>, kTileBytes, attr_v4_done);
            if (e != cudaSuccess)
                return e;
            planned_kernel_v4<TOD2MAP, RESP, PERIODIC><<<(unsigned) g, NT, kTileBytes, stream>>>(a, owner_mt, nowner,
                                                                                                 cellmap);
            return cudaGetLastError();
        }
    }
    static std::atomic<uint64_t> attr_done{0};
    cudaError_t e = set_smem_limit(planned_kernel<TOD2MAP, RESP, PERIODIC>, kTileBytes, attr_done);
    if (e != cudaSuccess)
        return e;
    planned_kernel<TOD2MAP, RESP, PERIODIC><<<(unsigned) g, NT, kTileBytes, stream>>>(a, owner_mt, nowner, cellmap);
    return cudaGetLastError();
}

template<bool TOD2MAP, bool RESP>
cudaError_t launch_planned_dispatch(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                    cudaStream_t stream)
{
    return a.periodic ? launch_planned_impl<TOD2MAP, RESP, true>(a, owner_mt, nowner, cellmap, stream)
                      : launch_planned_impl<TOD2MAP, RESP, false>(a, owner_mt, nowner, cellmap, stream);
}

template<bool TOD2MAP>
cudaError_t launch_unplanned_impl(const OpArgs &a, cudaStream_t stream)
{
    const bool aligned = ((((uintptr_t) a.xp) | ((uintptr_t) a.out) | ((uintptr_t) a.in)) & 15) == 0;
    const bool vec = aligned && ((a.nsamp & 3) == 0);
    const int64_t nvec = vec ? a.nsamp / 4 : a.nsamp;
    int64_t g = 8 * (int64_t) device_sm_count();
    g = std::max<int64_t>(1, std::min<int64_t>(g, (nvec + 255) / 256));
    if (vec)
        unplanned_kernel<TOD2MAP, 4><<<(unsigned) g, 256, 0, stream>>>(a);
    else
        unplanned_kernel<TOD2MAP, 1><<<(unsigned) g, 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_planned_map2tod(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   cudaStream_t stream)
{
    return a.response ? launch_planned_dispatch<false, true>(a, owner_mt, nowner, cellmap, stream)
                      : launch_planned_dispatch<false, false>(a, owner_mt, nowner, cellmap, stream);
}

cudaError_t launch_planned_tod2map(const OpArgs &a, const uint64_t *owner_mt, int64_t nowner, const uint32_t *cellmap,
                                   cudaStream_t stream)
{
    return a.response ? launch_planned_dispatch<true, true>(a, owner_mt, nowner, cellmap, stream)
                      : launch_planned_dispatch<true, false>(a, owner_mt, nowner, cellmap, stream);
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
