// extern "C" entry points of libgpu_mm_b200.so (declared in include/gpu_mm_b200.h).
//
// Argument checks restate check_arguments.cu:20-228 of the reference; error texts follow
// check_arguments.cu:42-58 so that the C++/Python layers raise the reference's messages.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>

#include "gmm_internal.hpp"

namespace gmm {

int device_sm_count()
{
    static int cache[128] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128)
        return 148;
    if (cache[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
        cache[dev] = n;
    }
    return cache[dev];
}

}  // namespace gmm

using namespace gmm;

namespace {

thread_local std::string g_last_error;

// Maximum radix digit width used by the plan sort; chosen by the autotuner (autotune.py) via
// gmm_set_sort_digit_bits, default 8.
int g_sort_max_digit_bits = 8;

constexpr int kSortGridMax = 320;
constexpr int64_t kCellmapBytes = (1 << 20) / 8;   // one bit per possible cell

int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where)
{
    std::ostringstream ss;
    ss << where << ": CUDA error: " << cudaGetErrorString(e);
    return fail(GMM_ERR_CUDA, ss.str());
}

int64_t align128(int64_t n) { return (n + 127) & ~127ll; }

// check_err (check_arguments.cu:42-58): first matching message wins.
int err_bits(uint32_t err, const char *where, uint32_t ignore)
{
    err &= ~ignore;
    if (err == 0)
        return 0;
    std::string w(where);
    if (err & GMM_ERR_BAD_YPIX)
        return fail((int) err, w + ": xpointing y-value is outside range [1,nypix_global-2].");
    if (err & GMM_ERR_BAD_XPIX)
        return fail((int) err, w + ": xpointing x-value is outside range, perhaps you want the 'periodic_xcoord' flag?");
    if (err & GMM_ERR_INCONSISTENT_NMT)
        return fail((int) err, w + ": inconsistent value of nmt between preplan/plan?! (should never happen)");
    if (err & GMM_ERR_NOT_IN_PIXELIZATION)
        return fail((int) err, w + ": xpointing (y,x) value is not in LocalPixelization (perhaps pixelization is too small, or you want the 'partial_pixelization' flag");
    return fail((int) err, w + ": bad errflags?! (should never happen)");
}

int check_nsamp(int64_t nsamp, const char *where)
{
    if ((nsamp <= 0) || (nsamp > (1ll << 31)) || (nsamp % 32) != 0) {
        std::ostringstream ss;
        ss << where << ": nsamp=" << nsamp << " must be positive, <= 2^31, and a multiple of 32";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return 0;
}

int check_npix(int64_t ny, int64_t nx, const char *where)
{
    if ((ny <= 0) || (ny > 64 * 1024) || (nx <= 0) || (nx > 64 * 1024)) {
        std::ostringstream ss;
        ss << where << ": nypix_global=" << ny << ", nxpix_global=" << nx << " must be in [1, 65536]";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    if (ny < 2 || nx < 2) {
        std::ostringstream ss;
        ss << where << ": nypix_global and nxpix_global must be >= 2 for bilinear interpolation";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return 0;
}

int check_lpix(const gmm_lpix *lp, const char *where)
{
    if (!lp || !lp->cell_offsets)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": null local pixelization");
    if (int rc = check_npix(lp->nypix_global, lp->nxpix_global, where))
        return rc;
    if ((lp->nycells <= 0) || (lp->nycells > 1024) || (lp->nxcells <= 0) || (lp->nxcells > 1024))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": nycells/nxcells must be in [1, 1024]");
    if ((lp->ystride <= 0) || (lp->ystride % 64) || (lp->polstride <= 0) || (lp->polstride % 64))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": ystride and polstride must be positive multiples of 64");
    return 0;
}

int check_ptr(const void *p, const char *where, const char *name)
{
    if (!p)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": null pointer '" + name + "'");
    return 0;
}

void geometry(int64_t nsamp, int64_t *nclpb, int64_t *nblocks)
{
    // PointingPrePlan.cu:162-165
    const int64_t ncl = (nsamp + 31) / 32;
    int64_t c = (ncl + GMM_PREPLAN_SIZE - 1) / GMM_PREPLAN_SIZE;
    c = (c > 16) ? c : 16;
    c = (c + 3) & ~3ll;
    *nclpb = c;
    *nblocks = (ncl + c - 1) / c;
}

int read_word(const uint32_t *dev, uint32_t *host, int n, cudaStream_t stream, const char *where)
{
    cudaError_t e = cudaMemcpyAsync(host, dev, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);
    return 0;
}

OpArgs make_args(const gmm_lpix *lp, const float *xp, int64_t nsamp, bool partial, bool accum, uint32_t *errword)
{
    OpArgs a;
    a.out = nullptr;
    a.in = nullptr;
    a.xp = xp;
    a.response = nullptr;
    a.ndet = 1;
    a.nperdet = nsamp;
    a.det_m = 0;
    a.det_sh1 = 0;
    a.det_sh2 = 0;
    a.cell_offsets = lp->cell_offsets;
    a.nsamp = nsamp;
    a.ny = lp->nypix_global;
    a.nx = lp->nxpix_global;
    a.periodic = lp->periodic_xcoord != 0;
    a.nycells = lp->nycells;
    a.nxcells = lp->nxcells;
    a.ystride = lp->ystride;
    a.polstride = lp->polstride;
    a.partial = partial;
    a.accum = accum;
    a.errword = errword;
    a.flush = kFlushF32;
    a.comp = nullptr;
    a.out64 = nullptr;
    a.max_run_lines = 0;
    a.hot_slot = nullptr;
    a.hot = nullptr;
    a.descs = nullptr;
    a.ntod = 0;
    a.ctas_per_sm = 0;
    a.min_lines_per_cta = 0;
    return a;
}

// Magic numbers for unsigned 32-bit division by d (Granlund & Montgomery 1994, round-up variant):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, q = (t + ((n - t) >> min(l,1))) >> max(l-1,0).
void set_divisor(OpArgs &a, uint32_t d)
{
    int l = 0;
    while ((1ull << l) < d) l++;
    a.det_m = (uint32_t) (((1ull << 32) * ((1ull << l) - d)) / d + 1);
    a.det_sh1 = std::min(l, 1);
    a.det_sh2 = std::max(l - 1, 0);
}

int check_plan_vs_lpix(const gmm_lpix *lp, const gmm_preplan_info *info, const char *where)
{
    // map2tod.cu:212-215
    if ((lp->nypix_global != info->nypix_global) || (lp->nxpix_global != info->nxpix_global) ||
        ((lp->periodic_xcoord != 0) != (info->periodic_xcoord != 0))) {
        std::ostringstream ss;
        ss << where << ": LocalPixelization (nypix_global=" << lp->nypix_global << ", nxpix_global="
           << lp->nxpix_global << ", periodic_xcoord=" << lp->periodic_xcoord << ") does not match plan (nypix_global="
           << info->nypix_global << ", nxpix_global=" << info->nxpix_global << ", periodic_xcoord="
           << info->periodic_xcoord << ")";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return 0;
}

}  // namespace

int gmm::report_err_bits(uint32_t err, const char *where, uint32_t ignore)
{
    return err_bits(err, where, ignore);
}

extern "C" {

const char *gmm_last_error(void) { return g_last_error.c_str(); }

// Records 'msg' as this thread's last error and returns 'code' (for the library's other files).
int gmm_fail_message(int code, const char *msg) { return fail(code, msg); }

const char *gmm_version(void) { return "gpu_mm_b200 0.1.0 (sm_100a)"; }

int gmm_set_sort_digit_bits(int32_t bits)
{
    if (bits < 4 || bits > 11)
        return fail(GMM_ERR_INVALID_ARGUMENT, "gmm_set_sort_digit_bits: bits must be in [4, 11]");
    g_sort_max_digit_bits = bits;
    return 0;
}

int gmm_get_sort_digit_bits(void) { return g_sort_max_digit_bits; }

int gmm_set_planned_tod2map_kernel(int32_t which)
{
    if ((which != GMM_TOD2MAP_BANDS) && (which != GMM_TOD2MAP_TILES))
        return fail(GMM_ERR_INVALID_ARGUMENT, "gmm_set_planned_tod2map_kernel: expected GMM_TOD2MAP_BANDS or GMM_TOD2MAP_TILES");
    g_tod2map_kernel = which;
    return 0;
}

int gmm_get_planned_tod2map_kernel(void) { return g_tod2map_kernel; }

// Passes and digit width of the owner-list sort of a single-TOD plan: by (cell, row band), kBandBits
// more key bits than the plan-word sort, with digits at most max(cell_dbits, kBandBits) wide (the sort
// scratch of gmm_preplan_info_init is sized for the wider of the two sorts).
static int owner_sort_passes(int nyc, int nxc, int cell_dbits, int *obits)
{
    return sort_passes(nyc, nxc, std::max(cell_dbits, kBandBits), obits, kBandBits);
}

int gmm_preplan_info_init(int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic, int64_t nmt, gmm_preplan_info *info)
{
    const char *where = "PointingPrePlan constructor";
    if (int rc = check_nsamp(nsamp, where)) return rc;
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (!info) return fail(GMM_ERR_INVALID_ARGUMENT, "gmm_preplan_info_init: null info");
    if ((nmt <= 0) || (nmt > (1ll << 30)))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": nmt out of range (0, 2^30]");

    std::memset(info, 0, sizeof(*info));
    int64_t nclpb, nblocks;
    geometry(nsamp, &nclpb, &nblocks);
    info->nsamp = nsamp;
    info->nypix_global = ny;
    info->nxpix_global = nx;
    info->periodic_xcoord = periodic ? 1 : 0;
    info->ncl_per_threadblock = nclpb;
    info->planner_nblocks = nblocks;
    info->plan_nmt = nmt;
    // PointingPrePlan.cu:236-238, 250
    int64_t nmt_per_tb = (int64_t) std::sqrt((double) nmt);
    nmt_per_tb = (nmt_per_tb + 32) & ~31ll;
    info->nmt_per_threadblock = nmt_per_tb;
    info->pointing_nblocks = (nmt + nmt_per_tb - 1) / nmt_per_tb;
    info->overhead = 32 * nmt / double(nsamp) - 1.0;

    int dbits = 0, obits = 0;
    sort_passes((ny + 63) / 64, (nx + 63) / 64, g_sort_max_digit_bits, &dbits);
    owner_sort_passes((ny + 63) / 64, (nx + 63) / 64, dbits, &obits);
    info->sort_digit_bits = dbits;
    info->sort_nbytes = sort_scratch_nbytes(std::max(dbits, obits), kSortGridMax);

    const int64_t ncl = nsamp / 32;
    const int64_t max_nblocks = std::max(info->planner_nblocks, info->pointing_nblocks);
    info->plan_nbytes = align128(8 * nmt) + align128(4 * max_nblocks) + align128(8 * ncl) + kCellmapBytes +
                        align128(8 * ncl);
    info->plan_constructor_tmp_nbytes = align128(8 * nmt) + align128(8 * ncl) + info->sort_nbytes;
    return 0;
}

int gmm_plan_layout_get(const gmm_preplan_info *info, gmm_plan_layout *layout)
{
    if (!info || !layout)
        return fail(GMM_ERR_INVALID_ARGUMENT, "gmm_plan_layout_get: null argument");
    const int64_t max_nblocks = std::max(info->planner_nblocks, info->pointing_nblocks);
    layout->mt_offset = 0;
    layout->err_offset = align128(8 * info->plan_nmt);
    layout->owner_offset = layout->err_offset + align128(4 * max_nblocks);
    layout->cellmap_offset = layout->owner_offset + align128(8 * (info->nsamp / 32));
    layout->band_offset = layout->cellmap_offset + kCellmapBytes;
    layout->total_nbytes = layout->band_offset + align128(8 * (info->nsamp / 32));
    return 0;
}

int gmm_preplan(const float *xp, int64_t nsamp, int32_t ny, int32_t nx, int32_t periodic, uint32_t *nmt_gpu,
                uint32_t *err_gpu, int32_t debug, cudaStream_t stream, gmm_preplan_info *info)
{
    (void) debug;
    const char *where = "PointingPrePlan constructor";
    if (int rc = check_nsamp(nsamp, where)) return rc;
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_ptr(xp, where, "xpointing")) return rc;
    if (int rc = check_ptr(nmt_gpu, where, "nmt_gpu")) return rc;
    if (int rc = check_ptr(err_gpu, where, "err_gpu")) return rc;
    if (int rc = check_ptr(info, where, "info")) return rc;

    int64_t nclpb, nblocks;
    geometry(nsamp, &nclpb, &nblocks);
    cudaError_t e = launch_preplan(xp, nsamp, ny, nx, periodic != 0, nclpb, (int) nblocks, nmt_gpu, err_gpu, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);
    uint32_t h[3] = {0, 0, 0};
    if (int rc = read_word(err_gpu, h, 3, stream, where)) return rc;
    if (int rc = err_bits(h[0], where, 0)) return rc;
    const int64_t nmt = (int64_t) h[1] | ((int64_t) h[2] << 32);
    if ((nmt <= 0) || (nmt > (1ll << 30))) {
        std::ostringstream ss;
        ss << where << ": nmt=" << nmt << " out of range (0, 2^30]";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return gmm_preplan_info_init(nsamp, ny, nx, periodic, nmt, info);
}

int gmm_plan_build(const gmm_preplan_info *info, const uint32_t *nmt_cumsum, const float *xp, void *buf,
                   int64_t buf_nbytes, void *tmp, int64_t tmp_nbytes, int32_t debug, cudaStream_t stream)
{
    (void) debug;
    const char *where = "PointingPlan constructor";
    if (int rc = check_ptr(info, where, "preplan")) return rc;
    if (int rc = check_ptr(nmt_cumsum, where, "nmt_cumsum")) return rc;
    if (int rc = check_ptr(xp, where, "xpointing")) return rc;
    if (int rc = check_ptr(buf, where, "buf")) return rc;
    if (int rc = check_ptr(tmp, where, "tmp_buf")) return rc;
    if (buf_nbytes < info->plan_nbytes || tmp_nbytes < info->plan_constructor_tmp_nbytes) {
        std::ostringstream ss;
        ss << where << ": expected 'buf' >= " << info->plan_nbytes << " bytes and 'tmp_buf' >= "
           << info->plan_constructor_tmp_nbytes << " bytes, got " << buf_nbytes << " and " << tmp_nbytes;
        return fail(GMM_ERR_BUFFER_TOO_SMALL, ss.str());
    }
    if ((((uintptr_t) buf) | ((uintptr_t) tmp)) & 127)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": 'buf' and 'tmp_buf' must be 128-byte aligned");

    gmm_plan_layout lay;
    gmm_plan_layout_get(info, &lay);
    char *b = (char *) buf;
    uint64_t *plan_mt = (uint64_t *) (b + lay.mt_offset);
    uint32_t *errflags = (uint32_t *) (b + lay.err_offset);
    uint64_t *owner = (uint64_t *) (b + lay.owner_offset);
    uint32_t *cellmap = (uint32_t *) (b + lay.cellmap_offset);
    uint64_t *band = (uint64_t *) (b + lay.band_offset);
    const int64_t nmt = info->plan_nmt, ncl = info->nsamp / 32;
    char *t = (char *) tmp;
    uint64_t *mt_alt = (uint64_t *) t;
    uint64_t *owner_alt = (uint64_t *) (t + align128(8 * nmt));
    uint32_t *hist = (uint32_t *) (t + align128(8 * nmt) + align128(8 * ncl));

    const int nyc = (info->nypix_global + 63) / 64, nxc = (info->nxpix_global + 63) / 64;
    int dbits = 0;
    const int passes = sort_passes(nyc, nxc, std::max(info->sort_digit_bits, 1), &dbits);
    if (dbits > info->sort_digit_bits && info->sort_digit_bits > 0)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": preplan sort digit width mismatch");
    const bool even = (passes % 2) == 0;
    int obits = 0;
    const int opasses = owner_sort_passes(nyc, nxc, dbits, &obits);
    const bool oeven = (opasses % 2) == 0;

    const int64_t err_nbytes = lay.owner_offset - lay.err_offset;
    cudaError_t e = cudaMemsetAsync(errflags, 0, err_nbytes, stream);
    if (e == cudaSuccess)
        e = launch_plan_emit(xp, info->nsamp, info->nypix_global, info->nxpix_global, info->periodic_xcoord != 0,
                             info->ncl_per_threadblock, (int) info->planner_nblocks, nmt_cumsum,
                             even ? plan_mt : mt_alt, oeven ? owner : owner_alt, band, errflags, stream);
    if (e == cudaSuccess)
        e = radix_sort_mt(even ? plan_mt : mt_alt, even ? mt_alt : plan_mt, nmt, nyc, nxc, dbits, passes, hist, stream);
    if (e == cudaSuccess)
        e = radix_sort_mt(oeven ? owner : owner_alt, oeven ? owner_alt : owner, ncl, nyc, nxc, obits, opasses, hist,
                          stream, 0, kBandBits);
    // Band words were written in line order; mt_alt (8 * nmt >= 8 * ncl bytes) is free after the sort
    // of plan_mt, so they go there and come back in owner-list order.
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mt_alt, band, 8 * ncl, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess)
        e = launch_band_gather(owner, ncl, mt_alt, band, stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(cellmap, 0, kCellmapBytes, stream);
    if (e == cudaSuccess)
        e = launch_plan_cellmap(plan_mt, nmt, cellmap, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);

    // check_gpu_errflags(err_gpu, planner_nblocks) (PointingPlan.cu:311)
    const int nb = (int) info->planner_nblocks;
    uint32_t h[GMM_PREPLAN_SIZE];
    if (int rc = read_word(errflags, h, nb, stream, where)) return rc;
    uint32_t err = 0;
    for (int i = 0; i < nb; i++)
        err |= h[i];
    return err_bits(err, where, 0);
}

// tod2map precision mode of planned_op (OpArgs::flush and friends).
struct Precision {
    int flush = kFlushF32;
    float *comp = nullptr;
    double *out64 = nullptr;
    int64_t max_run_lines = 0;
    const int32_t *hot_slot = nullptr;
    double *hot = nullptr;
};

static int planned_op(bool tod2map, float *out, const float *in, const float *xp, const float *response, int64_t ndet,
                      const gmm_lpix *lp, const gmm_preplan_info *info, const void *plan_buf, int32_t partial,
                      int32_t accum, uint32_t *errword, cudaStream_t stream, const char *where,
                      const Precision &prec = Precision())
{
    if (prec.flush == kFlushF64) {
        if (int rc = check_ptr(prec.out64, where, "local_map")) return rc;
    } else if (int rc = check_ptr(out, where, tod2map ? "local_map" : "tod")) {
        return rc;
    }
    if (prec.flush == kFlushCompensated) {
        if (int rc = check_ptr(prec.comp, where, "comp")) return rc;
    }
    if (prec.flush == kFlushHotF64) {
        if (int rc = check_ptr(prec.hot, where, "hot")) return rc;
        if (int rc = check_ptr(prec.hot_slot, where, "hot_slot")) return rc;
        if (((uintptr_t) in | (uintptr_t) xp) & 15)
            return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": tod and xpointing must be 16-byte aligned");
    }
    if (prec.max_run_lines < 0)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": max_run_lines must be >= 0");
    if (int rc = check_ptr(in, where, tod2map ? "tod" : "local_map")) return rc;
    if (int rc = check_ptr(xp, where, "xpointing")) return rc;
    if (int rc = check_ptr(info, where, "plan")) return rc;
    if (int rc = check_ptr(plan_buf, where, "plan buffer")) return rc;
    if (int rc = check_lpix(lp, where)) return rc;
    if (int rc = check_plan_vs_lpix(lp, info, where)) return rc;
    if (response) {
        if ((ndet <= 0) || (info->nsamp % ndet) != 0) {
            std::ostringstream ss;
            ss << where << ": response ndet=" << ndet << " must divide nsamp=" << info->nsamp;
            return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
        }
    }
    gmm_plan_layout lay;
    gmm_plan_layout_get(info, &lay);
    const char *b = (const char *) plan_buf;
    const uint64_t *owner = (const uint64_t *) (b + lay.owner_offset);
    const uint32_t *cellmap = (const uint32_t *) (b + lay.cellmap_offset);
    const uint64_t *band = (const uint64_t *) (b + lay.band_offset);
    uint32_t *word = errword ? errword : (uint32_t *) (b + lay.err_offset);

    OpArgs a = make_args(lp, xp, info->nsamp, partial != 0, accum != 0, word);
    a.out = out;
    a.in = in;
    a.flush = prec.flush;
    a.comp = prec.comp;
    a.out64 = prec.out64;
    a.max_run_lines = prec.max_run_lines;
    a.hot_slot = prec.hot_slot;
    a.hot = prec.hot;
    if (response) {
        a.response = response;
        a.ndet = ndet;
        a.nperdet = info->nsamp / ndet;
        set_divisor(a, (uint32_t) a.nperdet);
    }
    cudaError_t e = cudaMemsetAsync(word, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = tod2map ? launch_planned_tod2map(a, owner, info->nsamp / 32, cellmap, band, stream)
                    : launch_planned_map2tod(a, owner, info->nsamp / 32, cellmap, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);
    if (errword)
        return 0;
    uint32_t h = 0;
    if (int rc = read_word(word, &h, 1, stream, where)) return rc;
    return err_bits(h, where, partial ? GMM_ERR_NOT_IN_PIXELIZATION : 0);
}

int gmm_planned_map2tod(float *tod, const float *lmap, const float *xp, const gmm_lpix *lp, const gmm_preplan_info *info,
                        const void *plan_buf, int32_t partial, int32_t accum, uint32_t *errword, cudaStream_t stream)
{
    return planned_op(false, tod, lmap, xp, nullptr, 1, lp, info, plan_buf, partial, accum, errword, stream, "map2tod");
}

int gmm_planned_tod2map(float *lmap, const float *tod, const float *xp, const gmm_lpix *lp, const gmm_preplan_info *info,
                        const void *plan_buf, int32_t partial, uint32_t *errword, cudaStream_t stream)
{
    return planned_op(true, lmap, tod, xp, nullptr, 1, lp, info, plan_buf, partial, 0, errword, stream, "tod2map");
}

int gmm_response_map2tod(float *tod, const float *lmap, const float *xp, const float *response, int64_t ndet,
                         const gmm_lpix *lp, const gmm_preplan_info *info, const void *plan_buf, int32_t partial,
                         int32_t accum, uint32_t *errword, cudaStream_t stream)
{
    if (int rc = check_ptr(response, "response_map2tod", "response")) return rc;
    return planned_op(false, tod, lmap, xp, response, ndet, lp, info, plan_buf, partial, accum, errword, stream,
                      "map2tod");
}

int gmm_response_tod2map(float *lmap, const float *tod, const float *xp, const float *response, int64_t ndet,
                         const gmm_lpix *lp, const gmm_preplan_info *info, const void *plan_buf, int32_t partial,
                         uint32_t *errword, cudaStream_t stream)
{
    if (int rc = check_ptr(response, "response_tod2map", "response")) return rc;
    return planned_op(true, lmap, tod, xp, response, ndet, lp, info, plan_buf, partial, 0, errword, stream, "tod2map");
}

int gmm_planned_tod2map_compensated(float *lmap, float *comp, const float *tod, const float *xp, const gmm_lpix *lp,
                                    const gmm_preplan_info *info, const void *plan_buf, int32_t partial,
                                    int64_t max_run_lines, uint32_t *errword, cudaStream_t stream)
{
    Precision prec;
    prec.flush = kFlushCompensated;
    prec.comp = comp;
    prec.max_run_lines = max_run_lines;
    return planned_op(true, lmap, tod, xp, nullptr, 1, lp, info, plan_buf, partial, 0, errword, stream,
                      "tod2map_compensated", prec);
}

int gmm_planned_tod2map_f64(double *lmap, const float *tod, const float *xp, const gmm_lpix *lp,
                            const gmm_preplan_info *info, const void *plan_buf, int32_t partial, int64_t max_run_lines,
                            uint32_t *errword, cudaStream_t stream)
{
    Precision prec;
    prec.flush = kFlushF64;
    prec.out64 = lmap;
    prec.max_run_lines = max_run_lines;
    return planned_op(true, nullptr, tod, xp, nullptr, 1, lp, info, plan_buf, partial, 0, errword, stream,
                      "tod2map_f64", prec);
}

int gmm_plan_cell_lines(const gmm_preplan_info *info, const void *plan_buf, const gmm_lpix *lp, uint32_t *lines,
                        cudaStream_t stream)
{
    const char *where = "plan_cell_lines";
    if (int rc = check_ptr(info, where, "plan")) return rc;
    if (int rc = check_ptr(plan_buf, where, "plan buffer")) return rc;
    if (int rc = check_ptr(lines, where, "lines")) return rc;
    if (int rc = check_lpix(lp, where)) return rc;
    if (int rc = check_plan_vs_lpix(lp, info, where)) return rc;
    gmm_plan_layout lay;
    gmm_plan_layout_get(info, &lay);
    const uint64_t *mt = (const uint64_t *) ((const char *) plan_buf + lay.mt_offset);
    cudaError_t e = launch_plan_cell_lines(mt, info->plan_nmt, lp->nycells, lp->nxcells, lines, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

int gmm_hot_cells(const uint32_t *lines, const gmm_lpix *lp, uint32_t min_lines, int32_t *hot_slot, int32_t *hot_cells,
                  int32_t *nhot, cudaStream_t stream)
{
    const char *where = "hot_cells";
    if (int rc = check_ptr(lines, where, "lines")) return rc;
    if (int rc = check_ptr(hot_slot, where, "hot_slot")) return rc;
    if (int rc = check_ptr(hot_cells, where, "hot_cells")) return rc;
    if (int rc = check_ptr(nhot, where, "nhot")) return rc;
    if (int rc = check_lpix(lp, where)) return rc;
    cudaError_t e = launch_hot_cells(lines, lp->cell_offsets, lp->nycells * lp->nxcells, min_lines, hot_slot, hot_cells,
                                     nhot, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

int gmm_planned_tod2map_hot_f64(float *lmap, double *hot, const int32_t *hot_slot, const float *tod, const float *xp,
                                const gmm_lpix *lp, const gmm_preplan_info *info, const void *plan_buf, int32_t partial,
                                int64_t max_run_lines, uint32_t *errword, cudaStream_t stream)
{
    Precision prec;
    prec.flush = kFlushHotF64;
    prec.hot = hot;
    prec.hot_slot = hot_slot;
    prec.max_run_lines = max_run_lines;
    return planned_op(true, lmap, tod, xp, nullptr, 1, lp, info, plan_buf, partial, 0, errword, stream,
                      "tod2map_hot_f64", prec);
}

int gmm_fold_hot_f64(float *lmap, double *hot, const int32_t *hot_cells, int64_t nhot, const gmm_lpix *lp,
                     cudaStream_t stream)
{
    const char *where = "fold_hot_f64";
    if (int rc = check_ptr(lmap, where, "local_map")) return rc;
    if (nhot < 0)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": nhot must be >= 0");
    if (nhot == 0)
        return 0;
    if (int rc = check_ptr(hot, where, "hot")) return rc;
    if (int rc = check_ptr(hot_cells, where, "hot_cells")) return rc;
    if (int rc = check_lpix(lp, where)) return rc;
    if (nhot > (int64_t) lp->nycells * lp->nxcells)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": nhot exceeds the number of cells");
    cudaError_t e = launch_fold_hot(lmap, hot, hot_cells, nhot, lp->cell_offsets, lp->ystride, lp->polstride, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

int gmm_fold_compensation(float *lmap, float *comp, int64_t n, cudaStream_t stream)
{
    if (int rc = check_ptr(lmap, "fold_compensation", "local_map")) return rc;
    if (int rc = check_ptr(comp, "fold_compensation", "comp")) return rc;
    if (n < 0)
        return fail(GMM_ERR_INVALID_ARGUMENT, "fold_compensation: n must be >= 0");
    cudaError_t e = launch_fold_compensation(lmap, comp, n, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, "fold_compensation");
}

// ---- Batches of TODs ----

static int check_tuning(const gmm_batch_tuning *t, const char *where)
{
    if (!t) return 0;
    if ((t->sort_digit_bits < 4) || (t->sort_digit_bits > 11) || (t->ctas_per_sm < 1) || (t->ctas_per_sm > 8) ||
        (t->min_lines_per_cta < 1)) {
        std::ostringstream ss;
        ss << where << ": bad tuning (sort_digit_bits=" << t->sort_digit_bits << " in [4,11], ctas_per_sm="
           << t->ctas_per_sm << " in [1,8], min_lines_per_cta=" << t->min_lines_per_cta << " >= 1)";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return 0;
}

static int check_batch(const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, const char *where)
{
    if (int rc = check_ptr(descs, where, "descs")) return rc;
    if ((ntod < 1) || (ntod > 65535)) {
        std::ostringstream ss;
        ss << where << ": ntod=" << ntod << " must be in [1, 65535]";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    if ((total_lines < ntod) || (total_lines > (1ll << 40))) {
        std::ostringstream ss;
        ss << where << ": total_lines=" << total_lines << " must be >= ntod (every TOD has a cache line)";
        return fail(GMM_ERR_INVALID_ARGUMENT, ss.str());
    }
    return 0;
}

int gmm_batch_tuning_default(gmm_batch_tuning *tuning)
{
    if (int rc = check_ptr(tuning, "batch_tuning_default", "tuning")) return rc;
    tuning->sort_digit_bits = g_sort_max_digit_bits;
    tuning->ctas_per_sm = 2;
    tuning->min_lines_per_cta = 64;
    tuning->reserved = 0;
    return 0;
}

static void batch_layout(int64_t total_lines, int ny, int nx, const gmm_batch_tuning *t, int64_t *owner_off,
                         int64_t *cellmap_off, int64_t *plan_nbytes, int64_t *hist_off, int64_t *tmp_nbytes,
                         int *dbits, int *passes)
{
    const int nyc = (ny + 63) / 64, nxc = (nx + 63) / 64;
    *passes = sort_passes(nyc, nxc, t ? t->sort_digit_bits : g_sort_max_digit_bits, dbits);
    *owner_off = 0;
    *cellmap_off = align128(8 * total_lines);
    *plan_nbytes = *cellmap_off + kCellmapBytes;
    *hist_off = align128(8 * total_lines);
    *tmp_nbytes = *hist_off + std::max<int64_t>(sort_scratch_nbytes(*dbits, kSortGridMax), 128);
}

int gmm_batch_plan_nbytes(int64_t total_lines, int32_t ny, int32_t nx, const gmm_batch_tuning *tuning,
                          int64_t *plan_nbytes, int64_t *tmp_nbytes)
{
    const char *where = "batch_plan_nbytes";
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(plan_nbytes, where, "plan_nbytes")) return rc;
    if (int rc = check_ptr(tmp_nbytes, where, "tmp_nbytes")) return rc;
    if (total_lines < 1)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": total_lines must be >= 1");
    int64_t oo, co, ho;
    int dbits, passes;
    batch_layout(total_lines, ny, nx, tuning, &oo, &co, plan_nbytes, &ho, tmp_nbytes, &dbits, &passes);
    return 0;
}

int gmm_batch_plan_build(const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, int32_t ny, int32_t nx,
                         int32_t periodic, void *plan_buf, int64_t plan_nbytes, void *tmp, int64_t tmp_nbytes,
                         const gmm_batch_tuning *tuning, uint32_t *errword, cudaStream_t stream)
{
    const char *where = "batch_plan_build";
    if (int rc = check_batch(descs, ntod, total_lines, where)) return rc;
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(plan_buf, where, "plan_buf")) return rc;
    if (int rc = check_ptr(tmp, where, "tmp")) return rc;
    if (int rc = check_ptr(errword, where, "errword")) return rc;
    if ((((uintptr_t) plan_buf) | ((uintptr_t) tmp)) & 127)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": 'plan_buf' and 'tmp' must be 128-byte aligned");
    int64_t oo, co, need_plan, ho, need_tmp;
    int dbits, passes;
    batch_layout(total_lines, ny, nx, tuning, &oo, &co, &need_plan, &ho, &need_tmp, &dbits, &passes);
    if ((plan_nbytes < need_plan) || (tmp_nbytes < need_tmp)) {
        std::ostringstream ss;
        ss << where << ": buffers too small (plan " << plan_nbytes << " < " << need_plan << " or tmp " << tmp_nbytes
           << " < " << need_tmp << ")";
        return fail(GMM_ERR_BUFFER_TOO_SMALL, ss.str());
    }
    char *b = (char *) plan_buf, *t = (char *) tmp;
    uint64_t *owner = (uint64_t *) (b + oo), *alt = (uint64_t *) t;
    uint32_t *cellmap = (uint32_t *) (b + co), *hist = (uint32_t *) (t + ho);
    const bool even = (passes % 2) == 0;
    const int nyc = (ny + 63) / 64, nxc = (nx + 63) / 64;
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(cellmap, 0, kCellmapBytes, stream);
    if (e == cudaSuccess)
        e = launch_batch_owner(descs, ntod, total_lines, ny, nx, periodic != 0, even ? owner : alt, cellmap, nullptr,
                               errword, stream);
    if (e == cudaSuccess)
        e = radix_sort_mt(even ? owner : alt, even ? alt : owner, total_lines, nyc, nxc, dbits, passes, hist, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

int gmm_batch_plan_merge(const void *const *plans, const int64_t *nlines, int32_t ntod, int64_t total_lines,
                         int32_t ny, int32_t nx, void *plan_buf, int64_t plan_nbytes, void *tmp, int64_t tmp_nbytes,
                         const gmm_batch_tuning *tuning, cudaStream_t stream)
{
    const char *where = "batch_plan_merge";
    if (int rc = check_ptr(plans, where, "plans")) return rc;
    if (int rc = check_ptr(nlines, where, "nlines")) return rc;
    if ((ntod < 1) || (ntod > 65535) || (total_lines < ntod))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": need 1 <= ntod <= 65535 and total_lines >= ntod");
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(plan_buf, where, "plan_buf")) return rc;
    if (int rc = check_ptr(tmp, where, "tmp")) return rc;
    if ((((uintptr_t) plan_buf) | ((uintptr_t) tmp)) & 127)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": 'plan_buf' and 'tmp' must be 128-byte aligned");
    int64_t oo, co, need_plan, ho, need_tmp;
    int dbits, passes;
    batch_layout(total_lines, ny, nx, tuning, &oo, &co, &need_plan, &ho, &need_tmp, &dbits, &passes);
    if ((plan_nbytes < need_plan) || (tmp_nbytes < need_tmp))
        return fail(GMM_ERR_BUFFER_TOO_SMALL, std::string(where) + ": buffers too small");
    char *b = (char *) plan_buf, *t = (char *) tmp;
    uint64_t *owner = (uint64_t *) (b + oo), *alt = (uint64_t *) t;
    uint32_t *cellmap = (uint32_t *) (b + co), *hist = (uint32_t *) (t + ho);
    const bool even = (passes % 2) == 0;
    const int nyc = (ny + 63) / 64, nxc = (nx + 63) / 64;
    cudaError_t e = cudaMemsetAsync(cellmap, 0, kCellmapBytes, stream);
    if (e == cudaSuccess)
        e = launch_batch_merge(plans, nlines, ntod, total_lines, even ? owner : alt, cellmap, stream);
    if (e == cudaSuccess)
        e = radix_sort_mt(even ? owner : alt, even ? alt : owner, total_lines, nyc, nxc, dbits, passes, hist, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

static int each_tod_bits(int32_t ntod)
{
    int b = 0;
    while ((1 << b) < ntod) b++;
    return b;
}

int gmm_batch_plan_each_tmp_nbytes(int64_t total_lines, int32_t ntod, int32_t ny, int32_t nx,
                                   const gmm_batch_tuning *tuning, int64_t *tmp_nbytes)
{
    const char *where = "batch_plan_each_tmp_nbytes";
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(tmp_nbytes, where, "tmp_nbytes")) return rc;
    if ((ntod < 1) || (ntod > 4096) || (total_lines < ntod))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": need 1 <= ntod <= 4096 and total_lines >= ntod");
    int dbits = 0;
    sort_passes((ny + 63) / 64, (nx + 63) / 64, tuning ? tuning->sort_digit_bits : g_sort_max_digit_bits, &dbits,
                each_tod_bits(ntod));
    *tmp_nbytes = 2 * align128(8 * total_lines) + std::max<int64_t>(sort_scratch_nbytes(dbits, kSortGridMax), 128);
    return 0;
}

int gmm_batch_plan_build_each(const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, int32_t ny, int32_t nx,
                              int32_t periodic, void *const *plans_gpu, void *tmp, int64_t tmp_nbytes,
                              const gmm_batch_tuning *tuning, uint32_t *errword, cudaStream_t stream)
{
    const char *where = "batch_plan_build_each";
    if (int rc = check_batch(descs, ntod, total_lines, where)) return rc;
    if (ntod > 4096)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": at most 4096 TODs per call");
    if (int rc = check_npix(ny, nx, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(plans_gpu, where, "plans")) return rc;
    if (int rc = check_ptr(tmp, where, "tmp")) return rc;
    if (int rc = check_ptr(errword, where, "errword")) return rc;
    if (((uintptr_t) tmp) & 127)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": 'tmp' must be 128-byte aligned");
    int64_t need = 0;
    if (int rc = gmm_batch_plan_each_tmp_nbytes(total_lines, ntod, ny, nx, tuning, &need)) return rc;
    if (tmp_nbytes < need)
        return fail(GMM_ERR_BUFFER_TOO_SMALL, std::string(where) + ": 'tmp' too small");
    const int tb = each_tod_bits(ntod);
    int dbits = 0;
    const int passes = sort_passes((ny + 63) / 64, (nx + 63) / 64,
                                   tuning ? tuning->sort_digit_bits : g_sort_max_digit_bits, &dbits, tb);
    char *t = (char *) tmp;
    uint64_t *a = (uint64_t *) t, *b = (uint64_t *) (t + align128(8 * total_lines));
    uint32_t *hist = (uint32_t *) (t + 2 * align128(8 * total_lines));
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = launch_plans_each(descs, ntod, total_lines, ny, nx, periodic != 0, plans_gpu, a, b, hist, dbits, passes, tb,
                              errword, stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

static int batch_op(bool tod2map, const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, float *lmap_out,
                    const float *lmap_in, const gmm_lpix *lp, const void *plan_buf, int32_t partial, int32_t accum,
                    const gmm_batch_tuning *tuning, uint32_t *errword, cudaStream_t stream, const char *where)
{
    if (int rc = check_batch(descs, ntod, total_lines, where)) return rc;
    if (int rc = check_lpix(lp, where)) return rc;
    if (int rc = check_tuning(tuning, where)) return rc;
    if (int rc = check_ptr(plan_buf, where, "plan_buf")) return rc;
    if (int rc = check_ptr(errword, where, "errword")) return rc;
    if (int rc = check_ptr(tod2map ? (const void *) lmap_out : (const void *) lmap_in, where, "local_map")) return rc;
    int64_t oo, co, pn, ho, tn;
    int dbits, passes;
    batch_layout(total_lines, lp->nypix_global, lp->nxpix_global, tuning, &oo, &co, &pn, &ho, &tn, &dbits, &passes);
    const char *b = (const char *) plan_buf;
    OpArgs a = make_args(lp, nullptr, 0, partial != 0, accum != 0, errword);
    a.out = lmap_out;
    a.in = lmap_in;
    a.descs = descs;
    a.ntod = ntod;
    if (tuning) {
        a.ctas_per_sm = tuning->ctas_per_sm;
        a.min_lines_per_cta = tuning->min_lines_per_cta;
    }
    cudaError_t e = cudaMemsetAsync(errword, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = tod2map ? launch_batch_tod2map(a, (const uint64_t *) (b + oo), total_lines, (const uint32_t *) (b + co), stream)
                    : launch_batch_map2tod(a, (const uint64_t *) (b + oo), total_lines, (const uint32_t *) (b + co), stream);
    return (e == cudaSuccess) ? 0 : cuda_fail(e, where);
}

int gmm_batch_map2tod(const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, const float *local_map,
                      const gmm_lpix *lp, const void *plan_buf, int32_t partial, int32_t accum,
                      const gmm_batch_tuning *tuning, uint32_t *errword, cudaStream_t stream)
{
    return batch_op(false, descs, ntod, total_lines, nullptr, local_map, lp, plan_buf, partial, accum, tuning, errword,
                    stream, "batch_map2tod");
}

int gmm_batch_tod2map(const gmm_tod_desc *descs, int32_t ntod, int64_t total_lines, float *local_map,
                      const gmm_lpix *lp, const void *plan_buf, int32_t partial, const gmm_batch_tuning *tuning,
                      uint32_t *errword, cudaStream_t stream)
{
    return batch_op(true, descs, ntod, total_lines, local_map, nullptr, lp, plan_buf, partial, 0, tuning, errword,
                    stream, "batch_tod2map");
}

static int unplanned_op(bool tod2map, float *out, const float *in, const float *xp, int64_t nsamp, const gmm_lpix *lp,
                        uint32_t *errflags, int64_t errflags_len, int32_t partial, int32_t accum, int32_t sync_check,
                        cudaStream_t stream, const char *where)
{
    if (int rc = check_nsamp(nsamp, where)) return rc;
    if (int rc = check_ptr(out, where, tod2map ? "local_map" : "tod")) return rc;
    if (int rc = check_ptr(in, where, tod2map ? "tod" : "local_map")) return rc;
    if (int rc = check_ptr(xp, where, "xpointing")) return rc;
    if (int rc = check_ptr(errflags, where, "errflags")) return rc;
    if (errflags_len < 1)
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": errflags must have length >= 1");
    if (int rc = check_lpix(lp, where)) return rc;
    OpArgs a = make_args(lp, xp, nsamp, partial != 0, accum != 0, errflags);
    a.out = out;
    a.in = in;
    cudaError_t e = cudaMemsetAsync(errflags, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = tod2map ? launch_unplanned_tod2map(a, stream) : launch_unplanned_map2tod(a, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);
    if (!sync_check)
        return 0;
    uint32_t h = 0;
    if (int rc = read_word(errflags, &h, 1, stream, where)) return rc;
    return err_bits(h, where, partial ? GMM_ERR_NOT_IN_PIXELIZATION : 0);
}

int gmm_unplanned_map2tod(float *tod, const float *lmap, const float *xp, int64_t nsamp, const gmm_lpix *lp,
                          uint32_t *errflags, int64_t errflags_len, int32_t partial, int32_t accum, int32_t sync_check,
                          cudaStream_t stream)
{
    return unplanned_op(false, tod, lmap, xp, nsamp, lp, errflags, errflags_len, partial, accum, sync_check, stream,
                        "unplanned_map2tod");
}

int gmm_unplanned_tod2map(float *lmap, const float *tod, const float *xp, int64_t nsamp, const gmm_lpix *lp,
                          uint32_t *errflags, int64_t errflags_len, int32_t partial, int32_t sync_check,
                          cudaStream_t stream)
{
    return unplanned_op(true, lmap, tod, xp, nsamp, lp, errflags, errflags_len, partial, 0, sync_check, stream,
                        "unplanned_tod2map");
}

int gmm_errword_read(const uint32_t *errword, uint32_t ignore, cudaStream_t stream)
{
    if (int rc = check_ptr(errword, "gmm_errword_read", "errword")) return rc;
    uint32_t h = 0;
    if (int rc = read_word(errword, &h, 1, stream, "gmm_errword_read")) return rc;
    return err_bits(h, "deferred check", ignore);
}

int gmm_expand_dynamic_map(uint32_t *global_ncells, int64_t *cell_offsets, int32_t nycells, int32_t nxcells,
                           const uint64_t *plan_mt, int64_t nmt, uint32_t *ncells_out, cudaStream_t stream)
{
    const char *where = "expand_dynamic_map";
    if (int rc = check_ptr(global_ncells, where, "global_ncells")) return rc;
    if (int rc = check_ptr(cell_offsets, where, "cell_offsets")) return rc;
    if (int rc = check_ptr(plan_mt, where, "plan_mt")) return rc;
    if ((nycells <= 0) || (nycells > 1024) || (nxcells <= 0) || (nxcells > 1024))
        return fail(GMM_ERR_INVALID_ARGUMENT, std::string(where) + ": nycells/nxcells must be in [1, 1024]");
    cudaError_t e = launch_expand_dynamic_map(global_ncells, cell_offsets, nycells, nxcells, plan_mt, nmt, stream);
    if (e != cudaSuccess)
        return cuda_fail(e, where);
    uint32_t h = 0;
    if (int rc = read_word(global_ncells, &h, 1, stream, where)) return rc;
    if (ncells_out)
        *ncells_out = h;
    return 0;
}

}  // extern "C"
