// po_b200.cu — C ABI of the B200 (sm_100a) PO diffraction library.
//
// Data path of one call (replaces HandlerPO::HandleOrientationsToLocalGpu,
// reference src/cuda/GpuDiffraction.cu:4159-4778):
//   1. stage:    flat mbs_po_beams arrays -> HBM (one cudaMemcpyAsync each),
//                then po_pack_kernel builds the device records.
//   2. diffract: po_diffract_kernel (regular zenith rows) and po_pole_kernel
//                (polar rows) write one partial Mueller plane per orientation
//                chunk, no atomics.
//   3. reduce:   po_reduce_kernel adds the chunk partials in a fixed order
//                into the caller's accumulator (deterministic).
#include "mbs_po_b200.h"
#include "po_device.cuh"
#include "po_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace mbs;

namespace {

struct GridDev {
    int n_az = 0, n_zen = 0;
    double *st = nullptr, *ct = nullptr;      // [n_zen+1]
    double *sphi = nullptr, *cphi = nullptr;  // [n_az]
    double *vf = nullptr;                     // [n_az*(n_zen+1)*3]
    double *theta = nullptr;                  // [n_zen+1] zenith angles
    int8_t *row_kind = nullptr;               // [n_zen+1]
    int32_t *pole_rows = nullptr;             // [n_pole]
    int n_pole = 0;
    int n_general = 0;
};

// Launch shapes of the diffraction kernel: threads per CTA, directions per
// thread and the minimum resident CTAs per SM the register budget is cut
// for.  mbs_po_autotune times them on the caller's batch and keeps the
// fastest per precision; variant 0, the default (the drop-in does not
// autotune), is the fastest on the column and aggregate workloads.
struct Variant {
    int tpb, dpt, minb;
};
constexpr Variant kVariantsF32[] = {{128, 3, 3}, {64, 3, 5}, {64, 3, 6},
                                    {96, 2, 5}, {128, 2, 4}, {64, 3, 4}};
constexpr Variant kVariantsF64[] = {{64, 3, 4}, {128, 1, 3}, {96, 2, 4}, {128, 1, 4}, {64, 2, 6}};
// Shapes of the kernels that also accumulate the no-shadow sums (the
// fastest of 128x2x4 / 128x3x3 / 64x2x6 / 128x2x3 for FP32C and 128x1x4 /
// 128x1x3 / 64x2x4 / 64x1x6 for FP64 on the column).
constexpr Variant kNoShadowF32 = {128, 3, 3};
constexpr Variant kNoShadowF64 = {128, 1, 3};
constexpr int kNumVariantsF32 = sizeof(kVariantsF32) / sizeof(Variant);
constexpr int kNumVariantsF64 = sizeof(kVariantsF64) / sizeof(Variant);

// One device allocation holding every per-batch array.
struct Arena {
    void *base = nullptr;
    size_t cap = 0;
};

}  // namespace

struct mbs_po_staged {
    Arena arena;
    DevBeam *beams = nullptr;
    DevVert *verts = nullptr;
    double *brec = nullptr;        // [kBrecWords][n_beams]
    double *vrec = nullptr;        // [kVrecWords][n_verts]
    double *moments = nullptr;
    int32_t *vbeg = nullptr;
    int32_t *beam_off = nullptr;
    double *weight = nullptr;
    int n_orient = 0;              // all instances: n_sets * orient_per_set
    int64_t n_beams = 0, n_verts = 0;
    int max_nv = 0;
    int n_sets = 1;                // output planes (size instances)
    int orient_per_set = 0;
    bool reused = false;           // re-filled by mbs_po_restage: grows like a context arena
};

struct mbs_po_ctx {
    int device = 0;
    // stream-ordered allocations of the growing scratch (partials, upload
    // area, re-filled staged batches) come from this context's own pool,
    // which keeps freed blocks (release threshold: never) instead of
    // returning them to the driver at every synchronisation: a growth step
    // then re-uses pool memory instead of mapping new pages
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;          // polar-row kernel, concurrent
    std::string err;
    bool has_grid = false, has_wave = false;
    GridDev grid;
    mbs_po_wave wave{};
    WaveConst wc{};
    // scratch
    double *partial = nullptr;
    size_t partial_cap = 0;      // doubles
    double *macc = nullptr;      // [2][G*16] device accumulators for host calls
    size_t macc_cap = 0;
    double *hres = nullptr;      // pinned [2][G*16]
    size_t hres_cap = 0;
    double *mfull = nullptr;     // [2][n_full*(n_zen+1)*16] interpolated planes (FFT-phi calls)
    size_t mfull_cap = 0;
    double *phiW = nullptr;      // azimuth interpolation weights [n_full][n_low]
    size_t phiW_cap = 0;
    int phiW_low = 0, phiW_full = 0;
    Arena raw;                   // raw upload area for staging
    int *d_status = nullptr;      // [0] pack status, [1] work counter of the diffraction kernel
    mbs_po_staged host_staged;   // reused by mbs_po_diffract
    cudaEvent_t ev[8] = {};
    cudaEvent_t partial_done = nullptr;   // recorded after each launch that used `partial`
    int variant[2] = {0, 0};     // chosen launch shape per precision
    // host-side phases of the last host call, ms (mbs_po_last_profile)
    double prof[8] = {};
};

namespace {

double host_ms()
{
    return std::chrono::duration<double, std::milli>(
        std::chrono::steady_clock::now().time_since_epoch()).count();
}

int fail(mbs_po_ctx *ctx, int code, const std::string &msg)
{
    if (ctx)
        ctx->err = msg;
    return code;
}

int cuda_fail(mbs_po_ctx *ctx, cudaError_t e, const char *where)
{
    return fail(ctx, MBS_PO_ECUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(expr, where)                                   \
    do {                                                  \
        cudaError_t e_ = (expr);                          \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
    } while (0)

template <typename T>
int ensure(mbs_po_ctx *ctx, T *&ptr, size_t &cap, size_t n, const char *what)
{
    if (n <= cap && ptr)
        return MBS_PO_OK;
    if (ptr)
        cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    const size_t alloc = std::max<size_t>(n, 1);
    cudaError_t e = cudaMalloc((void **)&ptr, alloc * sizeof(T));
    if (e != cudaSuccess)
        return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    cap = alloc;
    return MBS_PO_OK;
}

int ensure_arena(mbs_po_ctx *ctx, Arena &a, size_t bytes, const char *what)
{
    if (bytes <= a.cap && a.base)
        return MBS_PO_OK;
    cudaFree(a.base);
    a.base = nullptr;
    a.cap = 0;
    cudaError_t e = cudaMalloc(&a.base, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess)
        return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMalloc ") + what + ": " + cudaGetErrorString(e));
    a.cap = std::max<size_t>(bytes, 256);
    return MBS_PO_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// The orientation-chunk partials grow with the batch (more chunks) and are
// used on the caller's stream.  The old block is released in stream order on
// `st` after the last launch that used it (the partial_done event, recorded
// after each use on whatever stream that was), and the new one taken in
// stream order, at least twice the old size: a cudaFree here waits for all
// work on the device, in the reference's CLI the tracer threads' kernels too.
// The chunk partials grow to at least `min_doubles` at once: a first
// allocation sized for 64 chunk planes serves every call up to that many
// chunks (the drop-in's growing first batches among them) with one
// allocation instead of one per doubling (large device allocations on a
// busy host have taken up to 0.4 s each).
int grow_partial(mbs_po_ctx *ctx, size_t n, cudaStream_t st, size_t min_doubles = 0)
{
    if (n <= ctx->partial_cap && ctx->partial)
        return MBS_PO_OK;
    cudaError_t e = cudaSuccess;
    if (ctx->partial) {
        e = cudaStreamWaitEvent(st, ctx->partial_done, 0);
        if (e == cudaSuccess)
            e = cudaFreeAsync(ctx->partial, st);
        if (e != cudaSuccess)
            return fail(ctx, MBS_PO_ECUDA, std::string("releasing the partials: ") + cudaGetErrorString(e));
    }
    ctx->partial = nullptr;
    const size_t want = std::max<size_t>(std::max<size_t>(n, 2 * ctx->partial_cap), min_doubles);
    ctx->partial_cap = 0;
    e = cudaMallocFromPoolAsync((void **)&ctx->partial, want * sizeof(double), ctx->pool, st);
    if (e != cudaSuccess) {
        ctx->partial = nullptr;
        return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMallocAsync partials: ") + cudaGetErrorString(e));
    }
    ctx->partial_cap = want;
    return MBS_PO_OK;
}

// Context-owned arenas that are reused call after call (the upload area and
// the host entry points' staged batch).  Every earlier use of them has
// completed when they grow (stage_into and the host entry points end with a
// stream synchronisation), so the old block is released and the new one
// taken in stream order on `st`: unlike cudaFree, that waits for no other
// work on the device -- in the reference's CLI, tracer threads run their own
// kernels while a diffraction call stages its batch.  They grow to at least
// twice the request, four times the old size and 32 MiB, so batches that
// grow call by call (SelectGpuOrientationBatchSize doubles them) reallocate
// rarely: an allocation that has to grow the pool can wait for the device
// (up to 0.2 s in the reference CLI while its tracer threads run kernels).
int grow_arena(mbs_po_ctx *ctx, Arena &a, size_t bytes, const char *what, cudaStream_t st)
{
    if (bytes <= a.cap && a.base)
        return MBS_PO_OK;
    if (a.base) {
        cudaError_t e = cudaFreeAsync(a.base, st);
        if (e != cudaSuccess)
            return fail(ctx, MBS_PO_ECUDA, std::string("cudaFreeAsync ") + what + ": " + cudaGetErrorString(e));
    }
    a.base = nullptr;
    const size_t want = std::max<size_t>({(size_t)2 * bytes, (size_t)4 * a.cap, (size_t)32 << 20});
    const size_t cap = (want + ((size_t)1 << 21) - 1) & ~(((size_t)1 << 21) - 1);
    a.cap = 0;
    cudaError_t e = cudaMallocFromPoolAsync(&a.base, cap, ctx->pool, st);
    if (e != cudaSuccess) {
        a.base = nullptr;
        return fail(ctx, MBS_PO_ENOMEM, std::string("cudaMallocAsync ") + what + ": " + cudaGetErrorString(e));
    }
    a.cap = cap;
    return MBS_PO_OK;
}

void staged_release(mbs_po_staged *s)
{
    cudaFree(s->arena.base);
    *s = mbs_po_staged();
}

int validate(mbs_po_ctx *ctx, const mbs_po_beams *b)
{
    if (!b || b->n_orient < 0 || b->n_beams < 0 || b->n_verts < 0)
        return fail(ctx, MBS_PO_EINVAL, "null or negative-sized batch");
    if (b->n_beams >= (int64_t)1 << 31 || b->n_verts >= (int64_t)1 << 31)
        return fail(ctx, MBS_PO_ERANGE, "batch exceeds 2^31 beams or vertices");
    if (b->n_orient > 0 && (!b->beam_offsets || !b->orient_weight))
        return fail(ctx, MBS_PO_EINVAL, "missing orientation arrays");
    if (b->n_beams > 0 && (!b->vert_offsets || !b->vx || !b->vy || !b->slope_yx || !b->slope_xy
                           || !b->edge_flags || !b->beam_geom || !b->beam_flags))
        return fail(ctx, MBS_PO_EINVAL, "missing beam arrays");
    if (b->n_orient > 0 && (b->beam_offsets[0] != 0 || b->beam_offsets[b->n_orient] != b->n_beams))
        return fail(ctx, MBS_PO_EINVAL, "beam_offsets must run from 0 to n_beams");
    for (int o = 0; o < b->n_orient; ++o)
        if (b->beam_offsets[o + 1] < b->beam_offsets[o])
            return fail(ctx, MBS_PO_EINVAL, "beam_offsets not monotonic");
    if (b->n_beams > 0 && (b->vert_offsets[0] != 0 || b->vert_offsets[b->n_beams] != b->n_verts))
        return fail(ctx, MBS_PO_EINVAL, "vert_offsets must run from 0 to n_verts");
    for (int64_t i = 0; i < b->n_beams; ++i) {
        const int64_t nv = b->vert_offsets[i + 1] - b->vert_offsets[i];
        if (nv < 3 || nv > kMaxNv)
            return fail(ctx, MBS_PO_EBEAM, "beam " + std::to_string(i) + " has " + std::to_string(nv)
                                               + " vertices (valid edge data needs 3..31)");
    }
    return MBS_PO_OK;
}

void grid_release(GridDev &d)
{
    cudaFree(d.st); cudaFree(d.ct); cudaFree(d.sphi); cudaFree(d.cphi); cudaFree(d.vf);
    cudaFree(d.row_kind); cudaFree(d.pole_rows); cudaFree(d.theta);
    d = GridDev();
}

}  // namespace

// ------------------------------------------------------------------ C ABI --

extern "C" const char *mbs_po_version(void)
{
    return "mbs-b200 0.2 sm_100a (FP64 plain + FP32 compensated PO diffraction)";
}

extern "C" int mbs_po_create(mbs_po_ctx **out, int device)
{
    if (!out)
        return MBS_PO_EINVAL;
    *out = nullptr;
    mbs_po_ctx *ctx = new mbs_po_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
    for (int i = 0; i < 8 && e == cudaSuccess; ++i)
        e = cudaEventCreate(&ctx->ev[i]);
    if (e == cudaSuccess)
        e = cudaEventCreateWithFlags(&ctx->partial_done, cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&ctx->d_status, 64);
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        e = cudaMemPoolCreate(&ctx->pool, &props);
        uint64_t keep = ~(uint64_t)0;
        if (e == cudaSuccess)
            e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        if (ctx->pool)
            cudaMemPoolDestroy(ctx->pool);
        delete ctx;
        return MBS_PO_ECUDA;
    }
    *out = ctx;
    return MBS_PO_OK;
}

extern "C" int mbs_po_destroy(mbs_po_ctx *ctx)
{
    if (!ctx)
        return MBS_PO_EINVAL;
    cudaSetDevice(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if (ctx->side)
        cudaStreamSynchronize(ctx->side);
    grid_release(ctx->grid);
    cudaFree(ctx->partial);
    cudaFree(ctx->macc);
    cudaFree(ctx->mfull);
    cudaFree(ctx->phiW);
    cudaFreeHost(ctx->hres);
    cudaFree(ctx->raw.base);
    cudaFree(ctx->d_status);
    staged_release(&ctx->host_staged);
    for (int i = 0; i < 8; ++i)
        if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
    if (ctx->partial_done)
        cudaEventDestroy(ctx->partial_done);
    if (ctx->stream)
        cudaStreamDestroy(ctx->stream);
    if (ctx->side)
        cudaStreamDestroy(ctx->side);
    // staged batches the caller still holds keep their blocks; the pool's
    // resources go once the last of them is freed
    if (ctx->pool)
        cudaMemPoolDestroy(ctx->pool);
    delete ctx;
    return MBS_PO_OK;
}

extern "C" const char *mbs_po_last_error(const mbs_po_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : "null context";
}

extern "C" int mbs_po_set_grid(mbs_po_ctx *ctx, const mbs_po_grid *g)
{
    if (!ctx || !g || g->n_az <= 0 || g->n_zen < 0 || !g->theta || !g->vf)
        return fail(ctx, MBS_PO_EINVAL, "bad grid");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int nT = g->n_zen + 1, nAz = g->n_az;
    std::vector<double> st(nT), ct(nT), sphi(nAz), cphi(nAz);
    for (int t = 0; t < nT; ++t) {   // GpuDiffraction.cu:4536-4541
        st[t] = std::sin(g->theta[t]);
        ct[t] = std::cos(g->theta[t]);
    }
    for (int p = 0; p < nAz; ++p) {  // GpuDiffraction.cu:4543-4548
        const double phi = p * g->az_step;
        sphi[p] = std::sin(phi);
        cphi[p] = std::cos(phi);
    }
    // Zenith rows whose basis is not (-sin phi, cos phi, 0) are the polar
    // rows of ScatteringRange::ComputeSphereDirections (Handler.h:147-160).
    // When the basis and the direction are the same for every azimuth bin the
    // row is evaluated once (kind 1); otherwise per direction (kind 2).
    std::vector<int8_t> kind(nT, 0);
    std::vector<int32_t> poles;
    int nGeneral = 0;
    for (int t = 0; t < nT; ++t) {
        bool regular = true, same = true;
        const double *v0 = g->vf + (size_t)t * 3;
        for (int p = 0; p < nAz; ++p) {
            const double *v = g->vf + ((size_t)p * nT + t) * 3;
            if (std::fabs(v[0] + sphi[p]) + std::fabs(v[1] - cphi[p]) + std::fabs(v[2]) > 1e-12)
                regular = false;
            if (v[0] != v0[0] || v[1] != v0[1] || v[2] != v0[2])
                same = false;
        }
        if (regular)
            continue;
        if (same && std::fabs(st[t]) < 1e-12) {
            kind[t] = 1;
            poles.push_back(t);
        } else {
            kind[t] = 2;
            ++nGeneral;
        }
    }
    GridDev &d = ctx->grid;
    grid_release(d);
    const size_t nvf = (size_t)nAz * nT * 3;
    CK(cudaMalloc((void **)&d.st, nT * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.ct, nT * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.sphi, nAz * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.cphi, nAz * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.vf, nvf * sizeof(double)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.theta, nT * sizeof(double)), "cudaMalloc grid");
    CK(cudaMemcpy(d.theta, g->theta, nT * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMalloc((void **)&d.row_kind, nT * sizeof(int8_t)), "cudaMalloc grid");
    CK(cudaMalloc((void **)&d.pole_rows, std::max<size_t>(poles.size(), 1) * sizeof(int32_t)), "cudaMalloc grid");
    CK(cudaMemcpy(d.st, st.data(), nT * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.ct, ct.data(), nT * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.sphi, sphi.data(), nAz * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.cphi, cphi.data(), nAz * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.vf, g->vf, nvf * sizeof(double), cudaMemcpyHostToDevice), "grid copy");
    CK(cudaMemcpy(d.row_kind, kind.data(), nT * sizeof(int8_t), cudaMemcpyHostToDevice), "grid copy");
    if (!poles.empty())
        CK(cudaMemcpy(d.pole_rows, poles.data(), poles.size() * sizeof(int32_t), cudaMemcpyHostToDevice), "grid copy");
    d.n_az = nAz;
    d.n_zen = g->n_zen;
    d.n_pole = (int)poles.size();
    d.n_general = nGeneral;
    ctx->has_grid = true;
    return MBS_PO_OK;
}

extern "C" int mbs_po_set_wave(mbs_po_ctx *ctx, const mbs_po_wave *w)
{
    if (!ctx || !w || !(w->wave_index > 0.0))
        return fail(ctx, MBS_PO_EINVAL, "bad wave constants");
    ctx->wave = *w;
    WaveConst &c = ctx->wc;
    c.k = w->wave_index;
    c.cw_re = w->compl_wave_re;
    c.cw_im = w->compl_wave_im;
    c.icw_re = w->inv_compl_wave_re;
    c.icw_im = w->inv_compl_wave_im;
    c.eps1 = w->eps1;
    c.eps1_f32 = std::max(w->eps1, 3e-5);   // GpuDiffraction.cu:498-512
    c.wavelength = w->wavelength;
    c.ot_far_ref = w->ot_far_reference_path;
    c.ot_ping = w->ot_ping_distance;
    c.legacy_sign = w->legacy_sign;
    c.ot_phase_avg = w->ot_phase_average;
    ctx->has_wave = true;
    return MBS_PO_OK;
}

namespace {

// Upload a batch and build the device records into `s` (capacity reused).
// The records carry wave-dependent coefficients: a staged batch belongs to
// the wave constants set when it was staged.  With `scales` the batch is
// staged once per size factor (instance i = scales[i]); instance i's
// orientations are [i nO, (i+1) nO) and its results go to output set i.
int stage_into(mbs_po_ctx *ctx, const mbs_po_beams *b, mbs_po_staged *s, cudaStream_t st,
               const double *scales = nullptr, int n_scales = 0, double k_rephase = 0.0)
{
    int rc = validate(ctx, b);
    if (rc)
        return rc;
    if (!ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "wave constants must be set before staging");
    const int nI = scales ? n_scales : 1;
    if (scales) {
        if (n_scales < 1)
            return fail(ctx, MBS_PO_EINVAL, "no size scale factors");
        for (int i = 0; i < n_scales; ++i)
            if (!(scales[i] > 0.0) || !std::isfinite(scales[i]))
                return fail(ctx, MBS_PO_EINVAL, "size scale factors must be positive");
        if (b->n_beams > 0 && !b->beam_raw)
            return fail(ctx, MBS_PO_EINVAL, "size scaling needs the unphased Jones records (beam_raw)");
        if (b->n_beams > 0 && (b->abs_offsets == nullptr) != (b->abs_paths == nullptr)
            && b->abs_offsets && b->abs_offsets[b->n_beams] > 0)
            return fail(ctx, MBS_PO_EINVAL, "abs_offsets given without abs_paths");
    }
    if ((int64_t)nI * b->n_beams >= ((int64_t)1 << 31) || (int64_t)nI * b->n_verts >= ((int64_t)1 << 31)
        || (int64_t)nI * b->n_orient >= ((int64_t)1 << 31))
        return fail(ctx, MBS_PO_ERANGE, "staged instances exceed 2^31 beams, vertices or orientations");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int64_t nB = b->n_beams, nV = b->n_verts, nO = b->n_orient;
    const bool has_abs = scales && b->abs_offsets && b->abs_paths && nB > 0 && b->abs_offsets[nB] > 0;
    const int64_t nAbs = has_abs ? b->abs_offsets[nB] : 0;
    // raw upload area: vert_off, vx, vy, syx, sxy, geom, flags
    // (+ scales, raw Jones records, absorption paths for size instances)
    const size_t off_vo = 0;
    const size_t off_vx = off_vo + align256((nB + 1) * 8);
    const size_t off_vy = off_vx + align256(nV * 8);
    const size_t off_syx = off_vy + align256(nV * 8);
    const size_t off_sxy = off_syx + align256(nV * 8);
    const size_t off_g = off_sxy + align256(nV * 8);
    const size_t off_ef = off_g + align256(nB * MBS_PO_GEOM_STRIDE * 8);
    const size_t off_bf = off_ef + align256(nV);
    const size_t off_sc = off_bf + align256(nB);
    const size_t off_raw = off_sc + align256(scales ? nI * 8 : 0);
    const size_t off_ao = off_raw + align256(scales ? nB * MBS_PO_RAW_STRIDE * 8 : 0);
    const size_t off_ap = off_ao + align256(has_abs ? (nB + 1) * 8 : 0);
    const size_t raw_bytes = off_ap + align256(nAbs * 8);
    const double tg0 = host_ms();
    if ((rc = grow_arena(ctx, ctx->raw, raw_bytes, "staging", st)))
        return rc;
    unsigned char *raw = (unsigned char *)ctx->raw.base;
    // device records (nI instances)
    const int64_t iB = nI * nB, iV = nI * nV, iO = nI * nO;
    const size_t o_beams = 0;
    const size_t o_verts = o_beams + align256(iB * sizeof(DevBeam));
    const size_t o_brec = o_verts + align256(iV * sizeof(DevVert));
    const size_t o_vrec = o_brec + align256(iB * kBrecWords * sizeof(double));
    const size_t o_mom = o_vrec + align256(iV * kVrecWords * sizeof(double));
    const size_t o_vbeg = o_mom + align256(iB * kNumMoments * sizeof(double));
    const size_t o_boff = o_vbeg + align256((iB + 1) * sizeof(int32_t));
    const size_t o_w = o_boff + align256((iO + 1) * sizeof(int32_t));
    const size_t bytes = o_w + align256(std::max<int64_t>(iO, 1) * sizeof(double));
    if ((rc = (s == &ctx->host_staged || s->reused ? grow_arena(ctx, s->arena, bytes, "staged batch", st)
                                                   : ensure_arena(ctx, s->arena, bytes, "staged batch"))))
        return rc;
    const double tg1 = host_ms();
    ctx->prof[0] = tg1 - tg0;
    unsigned char *base = (unsigned char *)s->arena.base;
    s->beams = (DevBeam *)(base + o_beams);
    s->verts = (DevVert *)(base + o_verts);
    s->brec = (double *)(base + o_brec);
    s->vrec = (double *)(base + o_vrec);
    s->moments = (double *)(base + o_mom);
    s->vbeg = (int32_t *)(base + o_vbeg);
    s->beam_off = (int32_t *)(base + o_boff);
    s->weight = (double *)(base + o_w);

    std::vector<int32_t> boff(iO + 1);
    for (int i = 0; i < nI; ++i)
        for (int64_t o = 0; o < nO; ++o)
            boff[i * nO + o] = (int32_t)(i * nB + b->beam_offsets[o]);
    boff[iO] = (int32_t)iB;
    CK(cudaMemcpyAsync(s->beam_off, boff.data(), (iO + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, st), "H2D offsets");
    for (int i = 0; i < nI && nO > 0; ++i)
        CK(cudaMemcpyAsync(s->weight + i * nO, b->orient_weight, nO * sizeof(double), cudaMemcpyHostToDevice, st), "H2D weights");
    if (nB > 0) {
        CK(cudaMemcpyAsync(raw + off_vo, b->vert_offsets, (nB + 1) * 8, cudaMemcpyHostToDevice, st), "H2D vert_offsets");
        CK(cudaMemcpyAsync(raw + off_vx, b->vx, nV * 8, cudaMemcpyHostToDevice, st), "H2D vx");
        CK(cudaMemcpyAsync(raw + off_vy, b->vy, nV * 8, cudaMemcpyHostToDevice, st), "H2D vy");
        CK(cudaMemcpyAsync(raw + off_syx, b->slope_yx, nV * 8, cudaMemcpyHostToDevice, st), "H2D slope_yx");
        CK(cudaMemcpyAsync(raw + off_sxy, b->slope_xy, nV * 8, cudaMemcpyHostToDevice, st), "H2D slope_xy");
        CK(cudaMemcpyAsync(raw + off_g, b->beam_geom, nB * MBS_PO_GEOM_STRIDE * 8, cudaMemcpyHostToDevice, st), "H2D geom");
        CK(cudaMemcpyAsync(raw + off_ef, b->edge_flags, nV, cudaMemcpyHostToDevice, st), "H2D edge_flags");
        CK(cudaMemcpyAsync(raw + off_bf, b->beam_flags, nB, cudaMemcpyHostToDevice, st), "H2D beam_flags");
        if (scales) {
            CK(cudaMemcpyAsync(raw + off_sc, scales, nI * 8, cudaMemcpyHostToDevice, st), "H2D scales");
            CK(cudaMemcpyAsync(raw + off_raw, b->beam_raw, nB * MBS_PO_RAW_STRIDE * 8, cudaMemcpyHostToDevice, st), "H2D raw Jones");
            if (has_abs) {
                CK(cudaMemcpyAsync(raw + off_ao, b->abs_offsets, (nB + 1) * 8, cudaMemcpyHostToDevice, st), "H2D abs offsets");
                CK(cudaMemcpyAsync(raw + off_ap, b->abs_paths, nAbs * 8, cudaMemcpyHostToDevice, st), "H2D abs paths");
            }
        }
        CK(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st), "memset status");
        ctx->prof[1] = host_ms() - tg1;
        PackParams P;
        P.n_beams = nB;
        P.n_verts = nV;
        P.sc.scales = scales ? (const double *)(raw + off_sc) : nullptr;
        P.sc.raw = scales ? (const double *)(raw + off_raw) : nullptr;
        P.sc.abs_off = has_abs ? (const int64_t *)(raw + off_ao) : nullptr;
        P.sc.abs_paths = has_abs ? (const double *)(raw + off_ap) : nullptr;
        P.sc.k_rephase = k_rephase > 0.0 ? k_rephase : ctx->wc.k;
        P.sc.abs_coeff = ctx->wave.abs_coeff;
        P.vert_off = (const int64_t *)(raw + off_vo);
        P.vx = (const double *)(raw + off_vx);
        P.vy = (const double *)(raw + off_vy);
        P.syx = (const double *)(raw + off_syx);
        P.sxy = (const double *)(raw + off_sxy);
        P.eflags = raw + off_ef;
        P.geom = (const double *)(raw + off_g);
        P.bflags = raw + off_bf;
        P.wc = ctx->wc;
        P.beams = s->beams;
        P.verts = s->verts;
        P.brec = s->brec;
        P.vrec = s->vrec;
        P.brec_stride = iB;
        P.vrec_stride = iV;
        P.moments = s->moments;
        P.vbeg = s->vbeg;
        P.status = ctx->d_status;
        const int threads = 128;
        const dim3 blocks((unsigned)((nB + 1 + threads - 1) / threads), (unsigned)nI);
        po_pack_kernel<<<blocks, threads, 0, st>>>(P);
        CK(cudaGetLastError(), "pack kernel launch");
        int status = 0;
        CK(cudaMemcpyAsync(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H status");
        CK(cudaStreamSynchronize(st), "pack sync");
        ctx->prof[2] = host_ms() - tg1 - ctx->prof[1];
        if (status)
            return fail(ctx, MBS_PO_EBEAM, "malformed beam in batch");
    }
    s->n_orient = (int)iO;
    s->n_beams = iB;
    s->n_verts = iV;
    s->n_sets = nI;
    s->orient_per_set = (int)nO;
    int mx = 0;
    for (int64_t i = 0; i < nB; ++i)
        mx = std::max<int>(mx, (int)(b->vert_offsets[i + 1] - b->vert_offsets[i]));
    s->max_nv = mx;
    return MBS_PO_OK;
}

struct LaunchPlan {
    int tiles_per_row, n_chunks, orient_per_chunk, chunks_per_set;
};

// At most this many orientation chunks (partial Mueller planes) per set.
// The persistent kernel's last wave of work items leaves SMs idle; about 128
// items per resident CTA keep that tail near 0.5 % of the step (64 chunks:
// 1 % longer FP32C and FP64 steps on the column; 32: 3 %), at 256 planes of
// 11 MB on the headline grid.
constexpr int kMaxChunks = 256;

// Orientation chunks per output set: enough work items (chunk x azimuth x
// zenith tile) for about kMaxChunks / 2 per resident CTA of the persistent
// kernel, at most kMaxChunks chunks per set (each chunk owns a partial
// plane).  n_orient is per set; n_chunks counts all sets.

LaunchPlan plan_launch(int n_az, int n_t, int n_orient, int dirs_per_cta, int ctas_per_sm,
                       int n_sets = 1)
{
    LaunchPlan L;
    L.tiles_per_row = (n_t + dirs_per_cta - 1) / dirs_per_cta;
    const long long ctas_per_chunk = (long long)n_az * L.tiles_per_row;
    int sms = 148;
    {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess
            && cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && v > 0)
            sms = v;
    }
    n_sets = std::max(1, n_sets);
    const long long target = (long long)sms * ctas_per_sm * (kMaxChunks / 2);
    long long chunks = (target + ctas_per_chunk * n_sets - 1) / (ctas_per_chunk * n_sets);
    // at least 8 orientations per chunk: small calls (the drop-in's first,
    // growing batches) keep few partial planes, so the context's partial
    // buffer does not grow through many large allocations
    chunks = std::max<long long>(1, std::min<long long>(chunks, std::max(1, n_orient / 8)));
    chunks = std::min<long long>(chunks, kMaxChunks);
    L.orient_per_chunk = (int)((n_orient + chunks - 1) / chunks);
    L.chunks_per_set = (int)((n_orient + L.orient_per_chunk - 1) / std::max(1, L.orient_per_chunk));
    if (L.chunks_per_set < 1) L.chunks_per_set = 1;
    L.n_chunks = L.chunks_per_set * n_sets;
    return L;
}

// Persistent launch: as many CTAs as fit on the device at once (at most one
// per work item); P.work must be zero on `st` when the kernel starts.
template <typename T, int TPB, int DPT, bool NS, int MINB>
cudaError_t launch_one(const KParams &P, cudaStream_t st)
{
    auto kern = po_diffract_kernel<T, TPB, DPT, NS, MINB>;
    const size_t smem = diffract_smem_bytes<T, TPB, DPT, NS>();
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    int dev = 0, sms = 148, per_sm = 1;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess
        || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess
        || (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TPB, smem)) != cudaSuccess)
        return e;
    const int ctas = std::max(1, std::min(P.n_items, sms * std::max(per_sm, 1)));
    kern<<<ctas, TPB, smem, st>>>(P);
    return cudaGetLastError();
}

// The cases follow kVariantsF64 / kVariantsF32 entry by entry; no-shadow
// sums use kNoShadowF64 / kNoShadowF32.
cudaError_t launch_diffract(int precision, int variant, bool ns, const KParams &P, cudaStream_t st)
{
    if (precision == MBS_PO_FP64) {
        if (ns)
            return launch_one<double, 128, 1, true, 3>(P, st);
        switch (variant) {
        case 1: return launch_one<double, 128, 1, false, 3>(P, st);
        case 2: return launch_one<double, 96, 2, false, 4>(P, st);
        case 3: return launch_one<double, 128, 1, false, 4>(P, st);
        case 4: return launch_one<double, 64, 2, false, 6>(P, st);
        default: return launch_one<double, 64, 3, false, 4>(P, st);
        }
    }
    if (ns)
        return launch_one<float, 128, 3, true, 3>(P, st);
    switch (variant) {
    case 1: return launch_one<float, 64, 3, false, 5>(P, st);
    case 2: return launch_one<float, 64, 3, false, 6>(P, st);
    case 3: return launch_one<float, 96, 2, false, 5>(P, st);
    case 4: return launch_one<float, 128, 2, false, 4>(P, st);
    case 5: return launch_one<float, 64, 3, false, 4>(P, st);
    default: return launch_one<float, 128, 3, false, 3>(P, st);
    }
}

Variant shape_of(int pi, int variant, bool ns)
{
    if (ns)
        return pi == 0 ? kNoShadowF64 : kNoShadowF32;
    return pi == 0 ? kVariantsF64[variant] : kVariantsF32[variant];
}

int run_diffract(mbs_po_ctx *ctx, const mbs_po_staged *s, int precision, double *M_dev,
                 double *Mns_dev, cudaStream_t st, mbs_po_stats *stats, int variant = -1,
                 int orient_limit = -1)
{
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    if (precision != MBS_PO_FP64 && precision != MBS_PO_FP32C)
        return fail(ctx, MBS_PO_EINVAL, "unknown precision");
    const int nAz = ctx->grid.n_az, nT = ctx->grid.n_zen + 1;
    const int64_t G = (int64_t)nAz * nT;
    if (stats) {
        stats->launches = 0;
        stats->n_chunks = 0;
        stats->kernel_ms = stats->reduce_ms = 0.0;
        stats->beam_dir_evals = s->n_beams * G;
        stats->vert_dir_evals = s->n_verts * G;
    }
    if (s->n_orient == 0 || s->n_beams == 0 || G == 0)
        return MBS_PO_OK;
    const bool ns = Mns_dev != nullptr;
    const int pi = precision == MBS_PO_FP64 ? 0 : 1;
    if (variant < 0)
        variant = ctx->variant[pi];
    const Variant V = shape_of(pi, variant, ns);
    // the autotuner's slice: the first orient_limit orientations of set 0
    const int n_sets = orient_limit > 0 ? 1 : s->n_sets;
    const int per_set = orient_limit > 0 ? std::min(orient_limit, s->orient_per_set) : s->orient_per_set;
    const int n_orient = n_sets * per_set;
    const LaunchPlan L = plan_launch(nAz, nT, per_set, V.tpb * V.dpt, V.minb, n_sets);
    const size_t plane = (size_t)16 * G;
    int rc;
    if ((rc = grow_partial(ctx, plane * L.n_chunks * (ns ? 2 : 1), st, plane * 64 * (ns ? 2 : 1))))
        return rc;
    KParams P;
    P.beams = s->beams;
    P.verts = s->verts;
    P.brec = s->brec;
    P.vrec = s->vrec;
    P.brec_stride = s->n_beams;
    P.vrec_stride = s->n_verts;
    P.moments = s->moments;
    P.vbeg = s->vbeg;
    P.beam_off = s->beam_off;
    P.weight = s->weight;
    P.st = ctx->grid.st;
    P.ct = ctx->grid.ct;
    P.sphi = ctx->grid.sphi;
    P.cphi = ctx->grid.cphi;
    P.vf = ctx->grid.vf;
    P.row_kind = ctx->grid.row_kind;
    P.n_az = nAz;
    P.n_t = nT;
    P.n_orient = n_orient;
    P.orient_per_chunk = L.orient_per_chunk;
    P.tiles_per_row = L.tiles_per_row;
    P.orient_per_set = per_set;
    P.chunks_per_set = L.chunks_per_set;
    P.wc = ctx->wc;
    P.partial = ctx->partial;
    P.partial_ns = ns ? ctx->partial + plane * L.n_chunks : nullptr;
    P.work = ctx->d_status + 1;
    P.n_items = L.n_chunks * nAz * L.tiles_per_row;
    int launches = 0;
    CK(cudaEventRecord(ctx->ev[0], st), "event");
    // polar rows on the side stream, concurrently with the main kernel
    if (ctx->grid.n_pole > 0) {
        CK(cudaStreamWaitEvent(ctx->side, ctx->ev[0], 0), "side wait");
        dim3 pg((unsigned)L.n_chunks, (unsigned)ctx->grid.n_pole);
        if (ns)
            po_pole_kernel<true><<<pg, 256, 0, ctx->side>>>(P, ctx->grid.pole_rows);
        else
            po_pole_kernel<false><<<pg, 256, 0, ctx->side>>>(P, ctx->grid.pole_rows);
        CK(cudaGetLastError(), "pole kernel launch");
        CK(cudaEventRecord(ctx->ev[6], ctx->side), "event");
        ++launches;
    }
    CK(cudaMemsetAsync(P.work, 0, sizeof(int), st), "memset work counter");
    const cudaError_t e = launch_diffract(precision, variant, ns, P, st);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "diffraction kernel launch");
    ++launches;
    if (ctx->grid.n_pole > 0)
        CK(cudaStreamWaitEvent(st, ctx->ev[6], 0), "join side stream");
    CK(cudaEventRecord(ctx->ev[1], st), "event");
    const int rb = 256;
    const dim3 rg((unsigned)((G * 16 + rb - 1) / rb), (unsigned)n_sets);
    po_reduce_kernel<<<rg, rb, 0, st>>>(ctx->partial, L.chunks_per_set, G, M_dev);
    CK(cudaGetLastError(), "reduce launch");
    ++launches;
    if (ns) {
        po_reduce_kernel<<<rg, rb, 0, st>>>(P.partial_ns, L.chunks_per_set, G, Mns_dev);
        CK(cudaGetLastError(), "reduce launch");
        ++launches;
    }
    CK(cudaEventRecord(ctx->partial_done, st), "event");
    CK(cudaEventRecord(ctx->ev[2], st), "event");
    if (stats) {
        CK(cudaEventSynchronize(ctx->ev[2]), "event sync");
        float a = 0, b2 = 0;
        cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&b2, ctx->ev[1], ctx->ev[2]);
        stats->kernel_ms = a;
        stats->reduce_ms = b2;
        stats->launches = launches;
        stats->n_chunks = L.n_chunks;
    }
    return MBS_PO_OK;
}

}  // namespace

extern "C" int mbs_po_autotune(mbs_po_ctx *ctx, const mbs_po_staged *s, int precision,
                               int max_orient, int *best, double *ms_out, int ms_len)
{
    if (!ctx || !s || (precision != MBS_PO_FP64 && precision != MBS_PO_FP32C))
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int pi = precision == MBS_PO_FP64 ? 0 : 1;
    const int nv = pi == 0 ? kNumVariantsF64 : kNumVariantsF32;
    const int64_t G = (int64_t)ctx->grid.n_az * (ctx->grid.n_zen + 1);
    double *acc = nullptr;
    CK(cudaMalloc((void **)&acc, G * 16 * sizeof(double)), "cudaMalloc autotune");
    int bestv = 0;
    double bestms = 1e300;
    for (int v = 0; v < nv; ++v) {
        mbs_po_stats st;
        double ms = 0.0;
        for (int rep = 0; rep < 2; ++rep) {   // first run warms up
            const int rc = run_diffract(ctx, s, precision, acc, nullptr, ctx->stream, &st, v, max_orient);
            if (rc) {
                cudaFree(acc);
                return rc;
            }
            ms = st.kernel_ms;
        }
        if (ms_out && v < ms_len)
            ms_out[v] = ms;
        if (ms < bestms) {
            bestms = ms;
            bestv = v;
        }
    }
    cudaFree(acc);
    ctx->variant[pi] = bestv;
    if (best)
        *best = bestv;
    return MBS_PO_OK;
}

extern "C" int mbs_po_set_variant(mbs_po_ctx *ctx, int precision, int variant)
{
    if (!ctx || (precision != MBS_PO_FP64 && precision != MBS_PO_FP32C))
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    const int pi = precision == MBS_PO_FP64 ? 0 : 1;
    const int nv = pi == 0 ? kNumVariantsF64 : kNumVariantsF32;
    if (variant < 0 || variant >= nv)
        return fail(ctx, MBS_PO_ERANGE, "no such launch variant");
    ctx->variant[pi] = variant;
    return MBS_PO_OK;
}

extern "C" int mbs_po_stage(mbs_po_ctx *ctx, const mbs_po_beams *beams, mbs_po_staged **out)
{
    if (!ctx || !out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    *out = nullptr;
    mbs_po_staged *s = new mbs_po_staged();
    int rc = stage_into(ctx, beams, s, ctx->stream);
    if (rc) {
        staged_release(s);
        delete s;
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        staged_release(s);
        delete s;
        return cuda_fail(ctx, e, "stage sync");
    }
    *out = s;
    return MBS_PO_OK;
}

extern "C" int mbs_po_restage(mbs_po_ctx *ctx, const mbs_po_beams *beams, mbs_po_staged *s)
{
    if (!ctx)
        return MBS_PO_EINVAL;
    if (!s || !beams)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    s->reused = true;
    int rc = stage_into(ctx, beams, s, ctx->stream);
    if (!rc) {
        const cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess)
            rc = cuda_fail(ctx, e, "restage sync");
    }
    if (rc) {   // nothing usable is left in it until the next successful restage
        s->n_orient = 0;
        s->n_beams = s->n_verts = 0;
        s->orient_per_set = 0;
        s->n_sets = 1;
    }
    return rc;
}

extern "C" int mbs_po_staged_free(mbs_po_ctx *ctx, mbs_po_staged *s)
{
    if (!s)
        return MBS_PO_EINVAL;
    if (ctx)
        cudaSetDevice(ctx->device);
    staged_release(s);
    delete s;
    return MBS_PO_OK;
}

extern "C" int mbs_po_stage_repeat(mbs_po_ctx *ctx, const mbs_po_staged *src, int n,
                                   const int32_t *orient_index, const double *weight,
                                   mbs_po_staged **out)
{
    if (out)
        *out = nullptr;
    if (!ctx || !src || !out || n < 0 || (n > 0 && (!orient_index || !weight)))
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    if (src->n_sets != 1)
        return fail(ctx, MBS_PO_EINVAL, "multi-size staged batches cannot be repeated");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    // the source's orientation offsets, back on the host
    std::vector<int32_t> soff(src->n_orient + 1);
    CK(cudaMemcpy(soff.data(), src->beam_off, soff.size() * sizeof(int32_t), cudaMemcpyDeviceToHost),
       "D2H offsets");
    // consecutive entries whose ranges do not continue each other are
    // separated by a weight-0 orientation spanning [end, next begin): empty
    // when the next range starts at or before the end (a repeat), the
    // skipped beams (weighted 0) when it starts after it
    std::vector<int32_t> boff;
    std::vector<double> w;
    boff.reserve((size_t)n * 2 + 1);
    w.reserve((size_t)n * 2);
    for (int i = 0; i < n; ++i) {
        const int o = orient_index[i];
        if (o < 0 || o >= src->n_orient)
            return fail(ctx, MBS_PO_ERANGE, "orientation index outside the staged batch");
        if (!boff.empty() && boff.back() != soff[o]) {
            w.push_back(0.0);
            boff.push_back(soff[o]);
        } else if (boff.empty()) {
            boff.push_back(soff[o]);
        }
        w.push_back(weight[i]);
        boff.push_back(soff[o + 1]);
    }
    if (boff.empty())
        boff.push_back(0);
    if (w.size() >= ((size_t)1 << 31))
        return fail(ctx, MBS_PO_ERANGE, "repeated batch exceeds 2^31 orientations");
    mbs_po_staged *v = new mbs_po_staged();
    const size_t o_boff = 0, o_w = align256(boff.size() * sizeof(int32_t));
    int rc = ensure_arena(ctx, v->arena, o_w + std::max<size_t>(w.size(), 1) * sizeof(double), "repeated batch");
    if (rc) {
        delete v;
        return rc;
    }
    unsigned char *base = (unsigned char *)v->arena.base;
    v->beams = src->beams;
    v->verts = src->verts;
    v->brec = src->brec;
    v->vrec = src->vrec;
    v->moments = src->moments;
    v->vbeg = src->vbeg;
    v->beam_off = (int32_t *)(base + o_boff);
    v->weight = (double *)(base + o_w);
    v->n_orient = (int)w.size();
    v->n_beams = src->n_beams;
    v->n_verts = src->n_verts;
    v->max_nv = src->max_nv;
    v->n_sets = 1;
    v->orient_per_set = v->n_orient;
    cudaError_t e = cudaMemcpy(v->beam_off, boff.data(), boff.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !w.empty())
        e = cudaMemcpy(v->weight, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        staged_release(v);
        delete v;
        return cuda_fail(ctx, e, "H2D repeated batch");
    }
    *out = v;
    return MBS_PO_OK;
}

extern "C" int mbs_po_diffract_staged(mbs_po_ctx *ctx, const mbs_po_staged *s, int precision,
                                      double *M_dev, double *Mns_dev, void *stream,
                                      mbs_po_stats *stats)
{
    if (!ctx || !s || !M_dev)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return run_diffract(ctx, s, precision, M_dev, Mns_dev, (cudaStream_t)stream, stats);
}

namespace {

// Host-buffer path shared by mbs_po_diffract and mbs_po_diffract_multisize:
// ------------------------------------------------ azimuth interpolation --
// The FFT-phi path of the reference (GpuDiffraction.cu:3206-3320,
// fft_upsample_phi_arr2d_impl and fft_phi_pad_kernel) computes a Mueller grid
// on n_low azimuth bins, takes the DFT of every (zenith row, element) series
// over azimuth, keeps the frequencies f = k for k <= n_low/2 and f = k - n_low
// above (the Nyquist bin of an even n_low at +n_low/2 only), scales by
// 1/n_low, zero-pads to n_full bins, transforms back and keeps the real part.
// For real input that is one linear map of the n_low samples,
//   out(p) = sum_m W[p][m] low(m),
//   W[p][m] = (1/n_low) sum_{f in F} cos(2 pi f (p/n_full - m/n_low)),
// which the device applies as a small matrix product.  With x = 2 pi r / D,
// r = (p n_low - m n_full) mod D, D = n_full n_low, the frequency sum has the
// closed forms  sin(n_low x/2) / sin(x/2)  (odd n_low) and
// sin(n_low x/2) cos(x/2) / sin(x/2)  (even n_low, the Nyquist term at +n_low/2),
// n_low at r = 0; every angle is reduced exactly in integers first.

constexpr int kMaxPhiLow = 4096;      // W row of one output azimuth in shared memory
constexpr int kMaxPhiFull = 65535;    // output azimuths run on grid.y

void phi_weights(int n_low, int n_full, std::vector<double> &W)
{
    W.assign((size_t)n_full * n_low, 0.0);
    const int64_t D = (int64_t)n_full * n_low;
    const bool even = (n_low % 2) == 0;
    for (int p = 0; p < n_full; ++p)
        for (int m = 0; m < n_low; ++m) {
            int64_t r = ((int64_t)p * n_low - (int64_t)m * n_full) % D;
            if (r < 0)
                r += D;
            double S;
            if (r == 0) {
                S = n_low;
            } else {
                // n_low x / 2 = pi r / n_full, reduced modulo 2 pi
                const double sn = std::sin(M_PI * (double)(r % (2 * (int64_t)n_full)) / n_full);
                // x / 2 = pi r / D in (0, pi): sin from the nearer end
                const int64_t rr = r <= D / 2 ? r : D - r;
                const double sh = std::sin(M_PI * (double)rr / (double)D);
                double ch = std::cos(M_PI * (double)rr / (double)D);
                if (r > D / 2)
                    ch = -ch;
                S = even ? sn * ch / sh : sn / sh;
            }
            W[(size_t)p * n_low + m] = S / n_low;
        }
}

int run_phi_interp(mbs_po_ctx *ctx, const double *low, int n_low, int n_rows, double *full,
                   int n_full, cudaStream_t st)
{
    if (n_low < 1 || n_rows < 1 || n_full < n_low)
        return fail(ctx, MBS_PO_EINVAL, "azimuth interpolation needs 1 <= n_low <= n_full and rows");
    if (n_low > kMaxPhiLow || n_full > kMaxPhiFull)
        return fail(ctx, MBS_PO_ERANGE, "azimuth interpolation supports n_low <= "
                    + std::to_string(kMaxPhiLow) + " and n_full <= " + std::to_string(kMaxPhiFull));
    int rc;
    if (ctx->phiW_low != n_low || ctx->phiW_full != n_full) {
        std::vector<double> W;
        phi_weights(n_low, n_full, W);
        if ((rc = ensure(ctx, ctx->phiW, ctx->phiW_cap, W.size(), "azimuth weights")))
            return rc;
        // the stream may still be reading an earlier table
        CK(cudaStreamSynchronize(st), "sync");
        CK(cudaMemcpy(ctx->phiW, W.data(), W.size() * sizeof(double), cudaMemcpyHostToDevice), "H2D weights");
        ctx->phiW_low = n_low;
        ctx->phiW_full = n_full;
    }
    const int64_t plane = (int64_t)n_rows * 16;
    const int tb = 256;
    const dim3 g((unsigned)((plane + tb - 1) / tb), (unsigned)n_full);
    po_phi_interp_kernel<<<g, tb, n_low * sizeof(double), st>>>(low, ctx->phiW, n_low, plane, full);
    CK(cudaGetLastError(), "azimuth interpolation launch");
    return MBS_PO_OK;
}

// stage (one size instance per scale, or the batch as is), diffract into
// device accumulators, copy back, add into the caller's planes.  n_full > 0
// (one size instance only): the planes are interpolated from the grid's
// n_az azimuth bins to n_full bins on the device first, and the caller's
// planes are [n_full][n_zen+1][16].
// With `view` set, nothing is added into M_accum / Mns_accum: view[0] (and
// view[1] when no-shadow sums are asked for by a non-null Mns_accum) receive
// pointers to the planes in the page-locked result buffer, or NULL when the
// batch holds nothing to add.
// With `pre` set, `beams` is ignored and the already staged batch `pre`
// (one output set) is diffracted: nothing is uploaded.
int diffract_host(mbs_po_ctx *ctx, const mbs_po_beams *beams, const double *scales, int n_scales,
                  double k_rephase, int precision, double *M_accum, double *Mns_accum,
                  mbs_po_stats *stats, int n_full = 0, const double **view = nullptr,
                  const mbs_po_staged *pre = nullptr)
{
    if (view) {
        view[0] = nullptr;
        view[1] = nullptr;
    }
    if (!ctx || (!beams && !pre) || !M_accum)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    if (scales && n_scales < 1)
        return fail(ctx, MBS_PO_EINVAL, "no size scale factors");
    if (pre && pre->n_sets != 1)
        return fail(ctx, MBS_PO_EINVAL, "multi-size staged batches use mbs_po_diffract_staged");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int64_t G = (int64_t)ctx->grid.n_az * (ctx->grid.n_zen + 1);
    if (pre ? (pre->n_orient == 0 || pre->n_beams == 0 || G == 0)
            : (beams->n_orient == 0 || beams->n_beams == 0 || G == 0))
        return pre ? MBS_PO_OK : validate(ctx, beams);
    cudaStream_t st = ctx->stream;
    const bool ns = Mns_accum != nullptr;
    const size_t sets = scales ? (size_t)n_scales : 1;
    const size_t n = (size_t)G * 16 * sets;
    const int n_rows = ctx->grid.n_zen + 1;
    // planes handed back: the grid's, or the interpolated ones
    const size_t n_out = n_full > 0 ? (size_t)n_full * n_rows * 16 : n;
    int rc;
    if ((rc = ensure(ctx, ctx->macc, ctx->macc_cap, n * 2, "accumulators")))
        return rc;
    if (n_full > 0 && (rc = ensure(ctx, ctx->mfull, ctx->mfull_cap, n_out * 2, "interpolated planes")))
        return rc;
    if (ctx->hres_cap < n_out * 2 || !ctx->hres) {
        cudaFreeHost(ctx->hres);
        ctx->hres = nullptr;
        ctx->hres_cap = 0;
        CK(cudaMallocHost((void **)&ctx->hres, n_out * 2 * sizeof(double)), "cudaMallocHost");
        ctx->hres_cap = n_out * 2;
    }
    for (double &v : ctx->prof)
        v = 0.0;
    CK(cudaEventRecord(ctx->ev[3], st), "event");
    if (!pre && (rc = stage_into(ctx, beams, &ctx->host_staged, st, scales, n_scales, k_rephase)))
        return rc;
    const double td0 = host_ms();
    CK(cudaEventRecord(ctx->ev[4], st), "event");
    CK(cudaMemsetAsync(ctx->macc, 0, n * (ns ? 2 : 1) * sizeof(double), st), "memset acc");
    rc = run_diffract(ctx, pre ? pre : &ctx->host_staged, precision, ctx->macc, ns ? ctx->macc + n : nullptr,
                      st, stats);
    if (rc)
        return rc;
    const double *dev_out = ctx->macc;
    if (n_full > 0) {
        CK(cudaMemsetAsync(ctx->mfull, 0, n_out * (ns ? 2 : 1) * sizeof(double), st), "memset planes");
        if ((rc = run_phi_interp(ctx, ctx->macc, ctx->grid.n_az, n_rows, ctx->mfull, n_full, st)))
            return rc;
        if (ns && (rc = run_phi_interp(ctx, ctx->macc + n, ctx->grid.n_az, n_rows, ctx->mfull + n_out,
                                       n_full, st)))
            return rc;
        dev_out = ctx->mfull;
    }
    CK(cudaEventRecord(ctx->ev[5], st), "event");
    CK(cudaMemcpyAsync(ctx->hres, dev_out, n_out * (ns ? 2 : 1) * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    CK(cudaEventRecord(ctx->ev[7], st), "event");
    const double td1 = host_ms();
    CK(cudaStreamSynchronize(st), "sync");
    const double td2 = host_ms();
    ctx->prof[3] = td1 - td0;
    ctx->prof[4] = td2 - td1;
    float h2d = 0.f, d2h = 0.f;
    cudaEventElapsedTime(&h2d, ctx->ev[3], ctx->ev[4]);
    cudaEventElapsedTime(&d2h, ctx->ev[5], ctx->ev[7]);
    if (view) {
        view[0] = ctx->hres;
        view[1] = ns ? ctx->hres + n_out : nullptr;
    } else {
        for (size_t i = 0; i < n_out; ++i)
            M_accum[i] += ctx->hres[i];
        if (ns)
            for (size_t i = 0; i < n_out; ++i)
                Mns_accum[i] += ctx->hres[n_out + i];
    }
    ctx->prof[5] = host_ms() - td2;
    if (stats) {
        stats->h2d_ms = h2d;
        stats->d2h_ms = d2h;
        stats->launches += pre ? 0 : 1;   // pack kernel
    }
    return MBS_PO_OK;
}

}  // namespace

extern "C" int mbs_po_diffract(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                               double *M_accum, double *Mns_accum, mbs_po_stats *stats)
{
    return diffract_host(ctx, beams, nullptr, 0, 0.0, precision, M_accum, Mns_accum, stats);
}

extern "C" int mbs_po_diffract_pinned(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                                      const double **M_out, const double **Mns_out, mbs_po_stats *stats)
{
    if (M_out)
        *M_out = nullptr;
    if (Mns_out)
        *Mns_out = nullptr;
    if (!ctx)
        return MBS_PO_EINVAL;
    if (!M_out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    // a non-null dummy accumulator selects the no-shadow sums; nothing is
    // written through either in view mode
    double dummy = 0.0;
    const double *view[2] = {nullptr, nullptr};
    const int rc = diffract_host(ctx, beams, nullptr, 0, 0.0, precision, &dummy, Mns_out ? &dummy : nullptr,
                                 stats, 0, view);
    *M_out = view[0];
    if (Mns_out)
        *Mns_out = view[1];
    return rc;
}

extern "C" int mbs_po_last_profile(const mbs_po_ctx *ctx, double *ms, int n)
{
    if (!ctx || !ms || n < 0)
        return MBS_PO_EINVAL;
    for (int i = 0; i < n && i < 8; ++i)
        ms[i] = ctx->prof[i];
    return MBS_PO_OK;
}

extern "C" int mbs_po_diffract_staged_pinned(mbs_po_ctx *ctx, const mbs_po_staged *staged, int precision,
                                             const double **M_out, const double **Mns_out,
                                             mbs_po_stats *stats)
{
    if (M_out)
        *M_out = nullptr;
    if (Mns_out)
        *Mns_out = nullptr;
    if (!ctx)
        return MBS_PO_EINVAL;
    if (!M_out || !staged)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    double dummy = 0.0;
    const double *view[2] = {nullptr, nullptr};
    const int rc = diffract_host(ctx, nullptr, nullptr, 0, 0.0, precision, &dummy, Mns_out ? &dummy : nullptr,
                                 stats, 0, view, staged);
    *M_out = view[0];
    if (Mns_out)
        *Mns_out = view[1];
    return rc;
}

// ---------------------------------------------- drop-in host helpers --
// Pure functions behind the drop-in's environment knobs (the caller reads
// the environment and passes the strings), so their rules are testable on
// any host.

extern "C" int mbs_po_multi_devices(int work_count, int device_count, const char *multi,
                                    const char *multi_max, int under_mpi)
{
    // gpu_multi_device_count, GpuDiffraction.cu:595-626
    if (work_count <= 1)
        return 1;
    if (multi && multi[0] == '0' && multi[1] == '\0')
        return 1;
    if ((!multi || !*multi) && under_mpi)
        return 1;
    if (device_count <= 1)
        return 1;
    int limit = device_count;
    if (multi && *multi) {
        char *end = nullptr;
        const long v = std::strtol(multi, &end, 10);
        if (end && *end == '\0' && v > 0)
            limit = (int)std::min<long>(v, 1 << 20);
    }
    if (multi_max) {
        char *end = nullptr;
        const long v = std::strtol(multi_max, &end, 10);
        if (end && *end == '\0' && v > 0)
            limit = std::min(limit, (int)std::min<long>(v, 1 << 20));
    }
    return std::max(1, std::min(std::min(device_count, limit), work_count));
}

extern "C" void mbs_po_device_range(int start, int count, int n_devices, int dev, int *begin,
                                    int *sub_count)
{
    // GpuDiffraction.cu:4224-4226
    const int64_t b = start + (int64_t)count * dev / std::max(1, n_devices);
    const int64_t e = start + (int64_t)count * (dev + 1) / std::max(1, n_devices);
    if (begin)
        *begin = (int)b;
    if (sub_count)
        *sub_count = (int)(e - b);
}

extern "C" double mbs_po_eps1_override(double eps1, const char *value)
{
    // gpu_effective_eps1, GpuDiffraction.cu:498-512 (the FP32 floor of 3e-5
    // is applied by the kernels' own threshold)
    if (value) {
        char *end = nullptr;
        const double v = std::strtod(value, &end);
        if (end && end != value && *end == '\0' && v > 0.0)
            return v;
    }
    return eps1;
}

extern "C" int mbs_po_beam_stats(const mbs_po_beams *b, char *buf, int len)
{
    // the MBS_GPU_BEAM_STATS line of GpuDiffraction.cu:4354-4443
    if (!b || !buf || len <= 0)
        return MBS_PO_EINVAL;
    const int64_t nB = b->n_beams;
    const int nO = b->n_orient;
    size_t hist[33] = {};
    size_t ext = 0, in = 0, ex = 0, ey = 0, mn = (size_t)-1, mx = 0;
    for (int o = 0; o < nO; ++o) {
        const size_t c = (size_t)(b->beam_offsets[o + 1] - b->beam_offsets[o]);
        mn = std::min(mn, c);
        mx = std::max(mx, c);
    }
    for (int64_t i = 0; i < nB; ++i) {
        const int64_t v0 = b->vert_offsets[i], v1 = b->vert_offsets[i + 1];
        const int nv = (int)(v1 - v0);
        if (nv >= 0 && nv <= 32)
            ++hist[nv];
        if (b->beam_flags[i] & MBS_PO_BEAM_EXTERNAL) ++ext; else ++in;
        for (int64_t v = v0; v < v1; ++v) {
            ex += (b->edge_flags[v] & MBS_PO_EDGE_VALID_X) ? 1 : 0;
            ey += (b->edge_flags[v] & MBS_PO_EDGE_VALID_Y) ? 1 : 0;
        }
    }
    std::string line = "GPU beam stats orient=" + std::to_string(nO) + " beams=" + std::to_string(nB);
    char tmp[256];
    std::snprintf(tmp, sizeof(tmp),
                  " beams/orient min=%zu mean=%.3f max=%zu external=%zu internal=%zu "
                  "valid_edges_x/beams=%.3f valid_edges_y/beams=%.3f vertices:",
                  mn == (size_t)-1 ? 0 : mn, nB == 0 ? 0.0 : (double)nB / (double)nO, mx, ext, in,
                  nB == 0 ? 0.0 : (double)ex / (double)nB, nB == 0 ? 0.0 : (double)ey / (double)nB);
    line += tmp;
    for (int nv = 1; nv <= 32; ++nv)
        if (hist[nv]) {
            std::snprintf(tmp, sizeof(tmp), " %d:%zu", nv, hist[nv]);
            line += tmp;
        }
    std::snprintf(buf, (size_t)len, "%s", line.c_str());
    return (int)line.size() < len ? MBS_PO_OK : MBS_PO_ERANGE;
}

extern "C" int mbs_po_diffract_fft_phi(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                                       int n_full, double *M_accum, double *Mns_accum,
                                       mbs_po_stats *stats)
{
    if (!ctx)
        return MBS_PO_EINVAL;
    if (ctx->has_grid && n_full < ctx->grid.n_az)
        return fail(ctx, MBS_PO_EINVAL, "n_full must be at least the grid's azimuth bins");
    return diffract_host(ctx, beams, nullptr, 0, 0.0, precision, M_accum, Mns_accum, stats, n_full);
}

extern "C" int mbs_po_phi_interpolate(mbs_po_ctx *ctx, const double *low_dev, int n_low, int n_rows,
                                      double *full_dev, int n_full, void *stream)
{
    if (!ctx || !low_dev || !full_dev)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    return run_phi_interp(ctx, low_dev, n_low, n_rows, full_dev, n_full, (cudaStream_t)stream);
}

extern "C" int mbs_po_diffract_multisize(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                                         const double *scales, int n_scales, double wave_index,
                                         int precision, double *M_accum, double *Mns_accum,
                                         mbs_po_stats *stats)
{
    if (!scales)
        return fail(ctx, MBS_PO_EINVAL, "null scales");
    return diffract_host(ctx, beams, scales, n_scales, wave_index, precision, M_accum, Mns_accum, stats);
}

extern "C" int mbs_po_stage_multisize(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                                      const double *scales, int n_scales, double wave_index,
                                      mbs_po_staged **out)
{
    if (!ctx || !out || !scales)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    *out = nullptr;
    mbs_po_staged *s = new mbs_po_staged();
    int rc = stage_into(ctx, beams, s, ctx->stream, scales, n_scales, wave_index);
    if (rc) {
        staged_release(s);
        delete s;
        return rc;
    }
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        staged_release(s);
        delete s;
        return cuda_fail(ctx, e, "stage sync");
    }
    *out = s;
    return MBS_PO_OK;
}

extern "C" int mbs_po_staged_sets(const mbs_po_staged *s)
{
    return s ? s->n_sets : 0;
}

extern "C" int mbs_po_phi_average(mbs_po_ctx *ctx, const double *M_dev, const double *dcos2pi,
                                  double *rows_out, double *csca_out, double *asym_out,
                                  void *stream)
{
    if (!ctx || !M_dev || !dcos2pi || !rows_out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_grid)
        return fail(ctx, MBS_PO_ESTATE, "grid must be set first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int nT = ctx->grid.n_zen + 1, nAz = ctx->grid.n_az;
    cudaStream_t st = (cudaStream_t)stream;
    double *buf = nullptr;
    size_t cap = 0;
    int rc;
    // [dcos2pi nT][rows nT*16][C_sca, g]
    if ((rc = ensure(ctx, buf, cap, (size_t)nT * 17 + 2, "azimuth average")))
        return rc;
    double *d_dc = buf, *d_rows = buf + nT, *d_out = d_rows + (size_t)nT * 16;
    cudaError_t e = cudaMemcpyAsync(d_dc, dcos2pi, nT * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        po_phi_average_kernel<<<nT, 128, 0, st>>>(M_dev, nAz, nT, ctx->grid.theta, d_rows);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        po_csca_kernel<<<1, 256, 0, st>>>(d_rows, nT, ctx->grid.theta, d_dc, d_out);
        e = cudaGetLastError();
    }
    double res[2] = {0.0, 0.0};
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(rows_out, d_rows, (size_t)nT * 16 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(res, d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "azimuth average");
    if (csca_out)
        *csca_out = res[0];
    if (asym_out)
        *asym_out = res[1];
    return MBS_PO_OK;
}

extern "C" int mbs_po_orientation_rows(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                                       double *rows_out)
{
    if (!ctx || !beams || (beams->n_orient > 0 && !rows_out))
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    int rc = validate(ctx, beams);
    if (rc)
        return rc;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int nO = beams->n_orient, nT = ctx->grid.n_zen + 1, nAz = ctx->grid.n_az;
    const size_t plane = (size_t)nAz * nT * 16;
    const size_t nrow = (size_t)nT * 16;
    std::memset(rows_out, 0, sizeof(double) * nrow * nO);
    if (nO == 0 || beams->n_beams == 0)
        return MBS_PO_OK;
    // orientation groups: one Mueller grid per orientation, at most 256 MiB
    // of grids per group, from the context's pool (stream-ordered: a later
    // call reuses the blocks without mapping new pages or synchronising)
    const int group = (int)std::max<size_t>(
        1, std::min<size_t>(std::min<size_t>(nO, 16384), ((size_t)1 << 25) / plane));
    double *grids = nullptr, *drows = nullptr;
    cudaStream_t st = ctx->stream;
    {
        cudaError_t e = cudaMallocFromPoolAsync((void **)&grids, plane * group * sizeof(double),
                                                ctx->pool, st);
        if (e == cudaSuccess)
            e = cudaMallocFromPoolAsync((void **)&drows, nrow * group * sizeof(double), ctx->pool, st);
        if (e != cudaSuccess) {
            if (grids)
                cudaFreeAsync(grids, st);
            return fail(ctx, MBS_PO_ENOMEM, std::string("orientation grids: ") + cudaGetErrorString(e));
        }
    }
    std::vector<int64_t> boff, voff;
    for (int o0 = 0; o0 < nO && rc == 0; o0 += group) {
        const int n = std::min(group, nO - o0);
        // the sub-batch [o0, o0+n) with rebased offsets
        const int64_t b0 = beams->beam_offsets[o0], b1 = beams->beam_offsets[o0 + n];
        const int64_t v0 = beams->vert_offsets[b0], v1 = beams->vert_offsets[b1];
        boff.resize(n + 1);
        for (int o = 0; o <= n; ++o)
            boff[o] = beams->beam_offsets[o0 + o] - b0;
        voff.resize(b1 - b0 + 1);
        for (int64_t b = b0; b <= b1; ++b)
            voff[b - b0] = beams->vert_offsets[b] - v0;
        mbs_po_beams sub = *beams;
        sub.n_orient = n;
        sub.n_beams = b1 - b0;
        sub.n_verts = v1 - v0;
        sub.beam_offsets = boff.data();
        sub.orient_weight = beams->orient_weight + o0;
        sub.vert_offsets = voff.data();
        sub.vx = beams->vx + v0;
        sub.vy = beams->vy + v0;
        sub.slope_yx = beams->slope_yx + v0;
        sub.slope_xy = beams->slope_xy + v0;
        sub.edge_flags = beams->edge_flags + v0;
        sub.beam_geom = beams->beam_geom + b0 * MBS_PO_GEOM_STRIDE;
        sub.beam_flags = beams->beam_flags + b0;
        sub.beam_raw = nullptr;
        sub.abs_offsets = nullptr;
        sub.abs_paths = nullptr;
        if ((rc = stage_into(ctx, &sub, &ctx->host_staged, st)))
            break;
        if (sub.n_beams == 0)
            continue;
        // every orientation its own output set
        ctx->host_staged.n_sets = n;
        ctx->host_staged.orient_per_set = 1;
        cudaError_t e = cudaMemsetAsync(grids, 0, plane * n * sizeof(double), st);
        if (e != cudaSuccess) {
            rc = cuda_fail(ctx, e, "memset grids");
            break;
        }
        if ((rc = run_diffract(ctx, &ctx->host_staged, precision, grids, nullptr, st, nullptr)))
            break;
        po_phi_average_kernel<<<dim3((unsigned)nT, (unsigned)n), 128, 0, st>>>(grids, nAz, nT,
                                                                               ctx->grid.theta, drows);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(rows_out + nrow * o0, drows, nrow * n * sizeof(double),
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            rc = cuda_fail(ctx, e, "orientation rows");
    }
    ctx->host_staged.n_sets = 1;
    cudaFreeAsync(grids, st);
    cudaFreeAsync(drows, st);
    return rc;
}

extern "C" int mbs_po_diffract_thetas(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                                      const double *theta_rad, int n, double *m11_out)
{
    if (!ctx || !beams || (n > 0 && (!theta_rad || !m11_out)) || n < 0)
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    if (n == 0)
        return validate(ctx, beams);
    for (int i = 0; i < n; ++i)
        m11_out[i] = 0.0;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t st = ctx->stream;
    int rc = stage_into(ctx, beams, &ctx->host_staged, st);
    if (rc)
        return rc;
    const mbs_po_staged &s = ctx->host_staged;
    if (s.n_beams == 0 || s.n_orient == 0)
        return MBS_PO_OK;
    // zenith angles clamped off the poles (GpuDiffraction.cu:4856-4866)
    constexpr double kPi = 3.14159265358979323846;
    std::vector<double> tab(2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        double th = theta_rad[i];
        if (th <= 1e-14)
            th = 1e-6;
        else if (th >= kPi - 1e-14)
            th = kPi - 1e-6;
        tab[i] = std::sin(th);
        tab[n + i] = std::cos(th);
    }
    const int nAz = ctx->grid.n_az;
    const int64_t pairs = s.n_beams * nAz;
    // chunks of about 64 (beam, azimuth) pairs per thread, at most 4096
    int64_t chunks = std::max<int64_t>(1, std::min<int64_t>(4096, pairs / (256 * 64)));
    const int bpc = (int)((s.n_beams + chunks - 1) / chunks);
    chunks = (s.n_beams + bpc - 1) / bpc;
    double *buf = nullptr;
    size_t cap = 0;
    const size_t need = 2 * (size_t)n + (size_t)chunks * n + n;
    if ((rc = ensure(ctx, buf, cap, need, "theta scan")))
        return rc;
    double *d_st = buf, *d_ct = buf + n, *part = buf + 2 * n, *d_m11 = part + (size_t)chunks * n;
    cudaError_t e = cudaMemcpyAsync(buf, tab.data(), 2 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        po_thetas_kernel<<<dim3((unsigned)n, (unsigned)chunks), 256, 0, st>>>(
            s.beams, s.verts, s.beam_off, s.weight, s.n_orient, s.n_beams, bpc, d_st, d_ct,
            ctx->grid.sphi, ctx->grid.cphi, nAz, n, ctx->wc, part);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        po_thetas_sum_kernel<<<(n + 127) / 128, 128, 0, st>>>(part, (int)chunks, n, d_m11);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(m11_out, d_m11, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "theta scan");
    return MBS_PO_OK;
}

extern "C" int mbs_po_extinction(mbs_po_ctx *ctx, const mbs_po_beams *beams, double *cext_out)
{
    if (!ctx || !beams || !cext_out)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "wave constants must be set first");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (beams->n_orient == 0)
        return MBS_PO_OK;
    cudaStream_t st = ctx->stream;
    int rc = stage_into(ctx, beams, &ctx->host_staged, st);
    if (rc)
        return rc;
    double *d = nullptr;
    size_t cap = 0;
    if ((rc = ensure(ctx, d, cap, (size_t)beams->n_orient, "cext")))
        return rc;
    const int th = 128;
    po_extinction_kernel<<<(beams->n_orient + th - 1) / th, th, 0, st>>>(
        ctx->host_staged.beams, ctx->host_staged.verts, ctx->host_staged.beam_off,
        ctx->host_staged.weight, beams->n_orient, ctx->wc, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cext_out, d, beams->n_orient * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "extinction");
    return MBS_PO_OK;
}

extern "C" int mbs_po_select_batch(mbs_po_ctx *ctx, const mbs_po_beams *beams, int start,
                                   int max_count, double mem_fraction, int *count_out)
{
    if (!ctx || !beams || !count_out || start < 0 || start > beams->n_orient)
        return fail(ctx, MBS_PO_EINVAL, "bad arguments");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    size_t freeB = 0, totalB = 0;
    CK(cudaMemGetInfo(&freeB, &totalB), "cudaMemGetInfo");
    if (!(mem_fraction > 0.1 && mem_fraction <= 0.98))
        mem_fraction = 0.88;   // MBS_GPU_MEM_FRACTION default (GpuDiffraction.cu:391-401)
    const int64_t G = ctx->has_grid ? (int64_t)ctx->grid.n_az * (ctx->grid.n_zen + 1) : 0;
    // fixed: partials (up to kMaxChunks chunks x 2 planes) + accumulators + 128 MiB slack
    const double fixed = (double)G * 16 * 8 * (kMaxChunks * 2 + 2) + (128.0 * (1 << 20));
    double budget = freeB * mem_fraction - fixed;
    int count = 0;
    const int end = std::min(beams->n_orient, start + std::max(0, max_count));
    const double per_beam = sizeof(DevBeam) + kBrecWords * 8 + kNumMoments * 8 + 4
                          + MBS_PO_GEOM_STRIDE * 8 + 8 + 1;
    const double per_vert = sizeof(DevVert) + kVrecWords * 8 + 4 * 8 + 1;
    for (int o = start; o < end; ++o) {
        const int64_t b0 = beams->beam_offsets[o], b1 = beams->beam_offsets[o + 1];
        const int64_t nv = b1 > b0 ? beams->vert_offsets[b1] - beams->vert_offsets[b0] : 0;
        const double need = (double)(b1 - b0) * per_beam + (double)nv * per_vert + 16;
        if (need > budget && count > 0)
            break;
        budget -= need;
        ++count;
    }
    *count_out = std::max(count, end > start ? 1 : 0);
    return MBS_PO_OK;
}

namespace {

// Best of three timed launches (after one warm-up) of a probe kernel of
// independent FMA chains, 16 x 8 FMAs per thread and iteration.
template <typename T>
int probe_peak(mbs_po_ctx *ctx, void (*kern)(T *, int, T, T), double *tflops)
{
    if (!ctx || !tflops)
        return MBS_PO_EINVAL;
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device);
    T *out = nullptr;
    const int blocks = sms * 8, threads = 256;
    const int iters = sizeof(T) == 4 ? 4096 : 2048;
    CK(cudaMalloc((void **)&out, (size_t)blocks * sizeof(T)), "cudaMalloc probe");
    double best = 0.0;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(ctx->ev[0], ctx->stream);
        kern<<<blocks, threads, 0, ctx->stream>>>(out, iters, (T)0.999999, (T)1e-6);
        cudaEventRecord(ctx->ev[1], ctx->stream);
        cudaError_t e = cudaEventSynchronize(ctx->ev[1]);
        if (e != cudaSuccess) {
            cudaFree(out);
            return cuda_fail(ctx, e, "probe");
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        if (rep > 0)
            best = std::max(best, flops / (ms * 1e-3) / 1e12);
    }
    cudaFree(out);
    *tflops = best;
    return MBS_PO_OK;
}

}  // namespace

extern "C" int mbs_po_probe_fp32_peak(mbs_po_ctx *ctx, double *tflops)
{
    return probe_peak<float>(ctx, po_fp32_probe_kernel, tflops);
}

extern "C" int mbs_po_probe_fp64_peak(mbs_po_ctx *ctx, double *tflops)
{
    return probe_peak<double>(ctx, po_fp64_probe_kernel, tflops);
}

// ------------------------------------------------- allocation-free variant --
// For callers that cannot allocate device memory at the time they diffract:
// callers whose device memory is owned by an external pool or a fixed budget
// that the library must not draw from, and real-time loops that must not
// block on cudaMalloc/cudaFree (both can synchronise the device).  mbs_po_diffract_staged keeps its chunk partials
// in context memory that it allocates and grows on demand; this variant
// keeps them in the fixed device array below instead.  The array is a
// file-scope __device__ variable, so every GPU that loads this library holds
// it (kNoAllocScratchBytes) until the process exits.

namespace {

constexpr size_t kNoAllocScratchBytes = MBS_PO_NOALLOC_SCRATCH_BYTES;
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
constexpr size_t kNoAllocHead = 32;   // work counter, 256 bytes

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch per device ordinal.  In host code the
// symbol is only a host-side stand-in, never a device address: it must be
// resolved with cudaGetSymbolAddress while that device is current.
constexpr int kMaxDevices = 64;
std::atomic<double *> g_noalloc_addr[kMaxDevices];

int noalloc_scratch(mbs_po_ctx *ctx, double **out)
{
    if (ctx->device < 0 || ctx->device >= kMaxDevices)
        return fail(ctx, MBS_PO_ERANGE, "device ordinal beyond the no-allocation table");
    double *addr = g_noalloc_addr[ctx->device].load();
    if (!addr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return cuda_fail(ctx, e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                             "cudaGetSymbolAddress(no-allocation scratch)");
        addr = static_cast<double *>(p);
        g_noalloc_addr[ctx->device].store(addr);
    }
    *out = addr;
    return MBS_PO_OK;
}

}  // namespace

extern "C" int mbs_po_diffract_staged_noalloc(mbs_po_ctx *ctx, const mbs_po_staged *s,
                                              int precision, double *M_dev, double *Mns_dev,
                                              void *stream)
{
    if (!ctx || !s || !M_dev)
        return fail(ctx, MBS_PO_EINVAL, "null argument");
    if (!ctx->has_grid || !ctx->has_wave)
        return fail(ctx, MBS_PO_ESTATE, "grid and wave constants must be set first");
    if (precision != MBS_PO_FP64 && precision != MBS_PO_FP32C)
        return fail(ctx, MBS_PO_EINVAL, "unknown precision");
    CK(cudaSetDevice(ctx->device), "cudaSetDevice");
    double *scratch = nullptr;
    int rc = noalloc_scratch(ctx, &scratch);
    if (rc)
        return rc;
    if (s->n_sets != 1)
        return fail(ctx, MBS_PO_EINVAL, "multi-size staged batches use mbs_po_diffract_staged");
    const int nAz = ctx->grid.n_az, nT = ctx->grid.n_zen + 1;
    const int64_t G = (int64_t)nAz * nT;
    if (s->n_orient == 0 || s->n_beams == 0 || G == 0)
        return MBS_PO_OK;
    const bool ns = Mns_dev != nullptr;
    const size_t plane = (size_t)16 * G;
    const size_t sets = ns ? 2 : 1;
    // the first kNoAllocHead doubles hold the work counter of the kernel
    int *work = reinterpret_cast<int *>(scratch);
    scratch += kNoAllocHead;
    // one partial plane per orientation chunk (and per output set) must fit
    if (plane * sets > kNoAllocScratchDoubles - kNoAllocHead)
        return fail(ctx, MBS_PO_ERANGE,
                    "grid of " + std::to_string(G) + " directions needs "
                    + std::to_string(plane * sets * sizeof(double)) + " bytes of partials; the "
                    "no-allocation scratch holds " + std::to_string(kNoAllocScratchBytes)
                    + " bytes (use mbs_po_diffract_staged)");
    const int pi = precision == MBS_PO_FP64 ? 0 : 1;
    const int variant = ctx->variant[pi];
    const Variant V = shape_of(pi, variant, ns);
    LaunchPlan L = plan_launch(nAz, nT, s->n_orient, V.tpb * V.dpt, V.minb);
    // fewer, larger orientation chunks when the fixed scratch is short
    const int max_chunks = (int)std::min<size_t>((kNoAllocScratchDoubles - kNoAllocHead) / (plane * sets), 64);
    if (L.n_chunks > max_chunks) {
        L.orient_per_chunk = (s->n_orient + max_chunks - 1) / max_chunks;
        L.n_chunks = (s->n_orient + L.orient_per_chunk - 1) / L.orient_per_chunk;
        L.chunks_per_set = L.n_chunks;
    }
    // Every partial entry of chunks [0, n_chunks) is written (not added) by
    // each call (first orientation of a chunk, polar rows), so the scratch
    // left by an earlier call needs no clearing.
    KParams P;
    P.beams = s->beams;
    P.verts = s->verts;
    P.brec = s->brec;
    P.vrec = s->vrec;
    P.brec_stride = s->n_beams;
    P.vrec_stride = s->n_verts;
    P.moments = s->moments;
    P.vbeg = s->vbeg;
    P.beam_off = s->beam_off;
    P.weight = s->weight;
    P.st = ctx->grid.st;
    P.ct = ctx->grid.ct;
    P.sphi = ctx->grid.sphi;
    P.cphi = ctx->grid.cphi;
    P.vf = ctx->grid.vf;
    P.row_kind = ctx->grid.row_kind;
    P.n_az = nAz;
    P.n_t = nT;
    P.n_orient = s->n_orient;
    P.orient_per_chunk = L.orient_per_chunk;
    P.tiles_per_row = L.tiles_per_row;
    P.orient_per_set = s->n_orient;
    P.chunks_per_set = L.n_chunks;
    P.wc = ctx->wc;
    P.partial = scratch;
    P.partial_ns = ns ? scratch + plane * L.n_chunks : nullptr;
    P.work = work;
    P.n_items = L.n_chunks * nAz * L.tiles_per_row;
    cudaStream_t st = (cudaStream_t)stream;
    if (ctx->grid.n_pole > 0) {
        CK(cudaEventRecord(ctx->ev[0], st), "event");
        CK(cudaStreamWaitEvent(ctx->side, ctx->ev[0], 0), "side wait");
        dim3 pg((unsigned)L.n_chunks, (unsigned)ctx->grid.n_pole);
        if (ns)
            po_pole_kernel<true><<<pg, 256, 0, ctx->side>>>(P, ctx->grid.pole_rows);
        else
            po_pole_kernel<false><<<pg, 256, 0, ctx->side>>>(P, ctx->grid.pole_rows);
        CK(cudaGetLastError(), "pole kernel launch");
        CK(cudaEventRecord(ctx->ev[6], ctx->side), "event");
    }
    CK(cudaMemsetAsync(work, 0, sizeof(int), st), "memset work counter");
    const cudaError_t e = launch_diffract(precision, variant, ns, P, st);
    if (e != cudaSuccess)
        return cuda_fail(ctx, e, "diffraction kernel launch");
    if (ctx->grid.n_pole > 0)
        CK(cudaStreamWaitEvent(st, ctx->ev[6], 0), "join side stream");
    const int rb = 256;
    const int rg = (int)((G * 16 + rb - 1) / rb);
    po_reduce_kernel<<<rg, rb, 0, st>>>(P.partial, L.n_chunks, G, M_dev);
    CK(cudaGetLastError(), "reduce launch");
    if (ns) {
        po_reduce_kernel<<<rg, rb, 0, st>>>(P.partial_ns, L.n_chunks, G, Mns_dev);
        CK(cudaGetLastError(), "reduce launch");
    }
    return MBS_PO_OK;
}
