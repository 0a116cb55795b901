// po_boundary.cpp — HandlerPO GPU entry points on top of the B200 library.
//
// This translation unit takes the place of the reference's CUDA backend TU
// (src/cuda/GpuDiffraction.cu) in the reference's own build: it defines the
// same HandlerPO member functions (declared in src/handler/HandlerPO.h:95-162)
// so that TracerPOTotal and the CLI call them unchanged.  Each call flattens
// the PreparedOrientation records (beam_pack.cpp) and calls the C ABI in
// include/mbs_po_b200.h.  Contracts kept from the reference:
//   - Mueller sums are added into localM / localM_noshadow (never
//     overwritten), rows p < nAz (GpuDiffraction.cu:4751-4766);
//   - incoherent mode and beams without valid edge data return false
//     (GpuDiffraction.cu:4172-4173, 4298-4303); the driver then throws;
//   - CUDA errors print "CUDA backend error at ..." and exit(2) unless
//     MBS_GPU_ALLOW_FALLBACK=1 (GpuDiffraction.cu:694-710);
//   - one context per host thread (thread_local, GpuDiffraction.cu:252).
// Environment knobs: MBS_B200_PRECISION=fp64|fp32c (default fp64, the
// reference's double build), MBS_GPU_TIMING=1 prints per-call timings,
// MBS_GPU_MEM_FRACTION bounds batch sizes like the reference; and the
// reference's own MBS_GPU_MULTI / MBS_GPU_MULTI_MAX (a call split over the
// visible devices, GpuDiffraction.cu:595-628, 4185-4270), MBS_GPU_EPS1 (the
// singular-edge threshold, :498-512) and MBS_GPU_BEAM_STATS=1 (per-batch
// beam statistics, :492-496, 4354-4443).  HandleOrientationsToLocalGpuOnDevice
// with a nonzero cacheToken keeps the staged beams on the device and reuses
// them for the next call with the same token and range (:3464-3500,
// 4276-4282).
#include "HandlerPO.h"
#include "FftStatistics.h"
#include "beam_pack.h"
#include "mbs_po_b200.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace
{

struct BoundaryContext
{
    mbs_po_ctx *ctx = nullptr;
    int device = -1;
    int gridNAz = -1, gridNZen = -1;
    std::vector<double> theta, vf;
    double azStep = 0.0;
    mbs_po_wave wave{};
    bool waveSet = false;
    std::vector<double> M, Mns;
    // the main path's packed batch, kept between calls so that its pages are
    // not allocated and first touched again on every call
    MbsPackedBeams packed;
    // packed-beam cache of HandleOrientationsToLocalGpuOnDevice: the staged
    // batch of (token, start, count) with the wave constants it was staged
    // under (its records hold them)
    mbs_po_staged *cached = nullptr;
    unsigned long long cachedToken = 0;
    int cachedStart = -1, cachedCount = -1;
    mbs_po_wave cachedWave{};

    ~BoundaryContext()
    {
        if (ctx)
        {
            if (cached)
                mbs_po_staged_free(ctx, cached);
            mbs_po_destroy(ctx);
        }
    }
};

thread_local BoundaryContext g_ctx;
// set on the multi-device split's workers and inside
// HandleOrientationsToLocalGpuOnDevice: no further split (g_gpuMultiWorker)
thread_local bool g_multiWorker = false;
// the OnDevice caller's packed-beam cache token (g_gpuPackCacheToken)
thread_local unsigned long long g_cacheToken = 0;

bool env_is(const char *name, const char *value)
{
    const char *v = std::getenv(name);
    return v && std::strcmp(v, value) == 0;
}

int precision_from_env()
{
    const char *v = std::getenv("MBS_B200_PRECISION");
    if (v && (std::strcmp(v, "fp32c") == 0 || std::strcmp(v, "fp32") == 0))
        return MBS_PO_FP32C;
    return MBS_PO_FP64;
}

bool report(int rc, const char *where)
{
    if (rc == MBS_PO_OK)
        return true;
    std::fprintf(stderr, "CUDA backend error at %s: %s\n", where,
                 g_ctx.ctx ? mbs_po_last_error(g_ctx.ctx) : "no context");
    if (!env_is("MBS_GPU_ALLOW_FALLBACK", "1"))
    {
        std::fprintf(stderr,
                     "FATAL: CUDA backend failed. Set MBS_GPU_ALLOW_FALLBACK=1 "
                     "to allow the legacy CPU fallback after GPU errors.\n");
        std::fflush(stderr);
        std::exit(2);
    }
    return false;
}

bool under_mpi()
{
    // gpu_running_under_mpi, GpuDiffraction.cu:574-592
    const char *names[] = {"OMPI_COMM_WORLD_SIZE", "PMI_SIZE", "PMIX_SIZE", "MPI_LOCALNRANKS"};
    for (const char *name : names)
    {
        const char *v = std::getenv(name);
        if (!v || !*v)
            continue;
        char *end = nullptr;
        const long n = std::strtol(v, &end, 10);
        if (end && *end == '\0' && n > 1)
            return true;
    }
    return false;
}

int multi_devices(int workCount)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess)
        count = 1;
    return mbs_po_multi_devices(workCount, count, std::getenv("MBS_GPU_MULTI"),
                                std::getenv("MBS_GPU_MULTI_MAX"), under_mpi() ? 1 : 0);
}

double mem_fraction()
{
    const char *v = std::getenv("MBS_GPU_MEM_FRACTION");
    if (!v || !*v)
        return 0.88;
    char *end = nullptr;
    const double p = std::strtod(v, &end);
    return (end && *end == '\0' && p > 0.1 && p <= 0.98) ? p : 0.88;
}

}  // namespace

// Shared set-up of one call: device context, grid tables and wave constants.
class HandlerPOBoundary
{
public:
    static bool Prepare(const HandlerPO &h, const ScatteringRange &sphere,
                        const mbs_po_wave &wave, int device)
    {
        BoundaryContext &c = g_ctx;
        if (c.ctx && c.device != device)
        {
            if (c.cached)
                mbs_po_staged_free(c.ctx, c.cached);
            c.cached = nullptr;
            c.cachedToken = 0;
            mbs_po_destroy(c.ctx);
            c.ctx = nullptr;
            c.gridNAz = c.gridNZen = -1;
            c.waveSet = false;
        }
        if (!c.ctx)
        {
            if (!report(mbs_po_create(&c.ctx, device), "context creation"))
                return false;
            c.device = device;
        }
        const int nAz = sphere.nAzimuth, nZen = sphere.nZenith;
        std::vector<double> theta(nZen + 1);
        for (int t = 0; t <= nZen; ++t)
            theta[t] = sphere.GetZenith(t);
        if (c.gridNAz != nAz || c.gridNZen != nZen || c.theta != theta
            || c.azStep != sphere.azinuthStep)
        {
            std::vector<double> vf((size_t)nAz * (nZen + 1) * 3);
            for (int p = 0; p < nAz; ++p)
                for (int t = 0; t <= nZen; ++t)
                {
                    const Point3d &v = sphere.vf[p][t];
                    double *o = &vf[((size_t)p * (nZen + 1) + t) * 3];
                    o[0] = v.x; o[1] = v.y; o[2] = v.z;
                }
            mbs_po_grid g;
            g.n_az = nAz;
            g.n_zen = nZen;
            g.az_step = sphere.azinuthStep;
            g.theta = theta.data();
            g.vf = vf.data();
            if (!report(mbs_po_set_grid(c.ctx, &g), "grid upload"))
                return false;
            c.gridNAz = nAz;
            c.gridNZen = nZen;
            c.theta.swap(theta);
            c.azStep = sphere.azinuthStep;
        }
        if (!c.waveSet || std::memcmp(&c.wave, &wave, sizeof(wave)) != 0)
        {
            if (!report(mbs_po_set_wave(c.ctx, &wave), "wave constants"))
                return false;
            c.wave = wave;
            c.waveSet = true;
        }
        (void)h;
        return true;
    }
};

// Wave constants of this handler; a subclass-free accessor to the protected
// Handler members through a pointer-to-member of a derived helper.
struct HandlerPOWaveAccess : public HandlerPO
{
    static mbs_po_wave Get(const HandlerPO &h, double waveIndexOverride)
    {
        mbs_po_wave w;
        std::memset(&w, 0, sizeof(w));
        w.wave_index = h.*(&HandlerPOWaveAccess::m_waveIndex);
        w.wavelength = h.*(&HandlerPOWaveAccess::m_wavelength);
        const complex cw = h.*(&HandlerPOWaveAccess::m_complWave);
        const complex icw = h.*(&HandlerPOWaveAccess::m_invComplWave);
        w.compl_wave_re = real(cw);
        w.compl_wave_im = imag(cw);
        w.inv_compl_wave_re = real(icw);
        w.inv_compl_wave_im = imag(icw);
        w.eps1 = mbs_po_eps1_override(h.*(&HandlerPOWaveAccess::m_eps1), std::getenv("MBS_GPU_EPS1"));
        w.abs_coeff = h.AbsorptionCoefficient();
        w.ot_far_reference_path = h.m_otFarReferencePath;
        w.ot_ping_distance = h.m_otPingDistance;
        w.legacy_sign = h.m_legacySign ? 1 : 0;
        w.ot_phase_average = h.m_otPhaseAverage ? 1 : 0;
        if (waveIndexOverride > 0.0)
        {
            // multi-size rescale: k is carried by the scale factor
            w.wave_index = waveIndexOverride;
        }
        return w;
    }
};

static int current_device()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        dev = 0;
    return dev;
}

// Adds a [n_az][n_rows][16] plane into the caller's Arr2D, whose cells are
// separate allocations (PhysMtr.cpp:6-17): one pass, azimuth rows spread over
// the OpenMP threads (serial when the caller is itself a parallel region).
static void add_plane(const double *plane, Arr2D &M, int nAz, int nRows)
{
#pragma omp parallel for schedule(static) if (nAz >= 8)
    for (int p = 0; p < nAz; ++p)
        for (int t = 0; t < nRows; ++t)
        {
            const double *m = plane + ((size_t)p * nRows + t) * 16;
            double *cell = M.RawCell(p, t);
            for (int q = 0; q < 16; ++q)
                cell[q] += m[q];
        }
}

// One device's share: packs prepared[start, start+count) (or reuses the
// staged beams of the OnDevice caller's cache token) and diffracts it on this
// thread's context; *Mv / *Mnv point at the sums in the context's page-locked
// result buffer (NULL when the range holds no beams), valid until this
// thread's next call.
static bool diffract_core(HandlerPO &h, const ScatteringRange &sphere,
                          const std::vector<PreparedOrientation> &prepared, int start, int count,
                          bool computeNoShadow, int device, const double **Mv, const double **Mnv)
{
    *Mv = *Mnv = nullptr;
    const bool timing = env_is("MBS_GPU_TIMING", "1");
    const auto t0 = std::chrono::steady_clock::now();
    const int nAz = sphere.nAzimuth, nZen = sphere.nZenith;
    const mbs_po_wave wave = HandlerPOWaveAccess::Get(h, 0.0);
    BoundaryContext &c = g_ctx;
    const unsigned long long token = g_cacheToken;
    const bool hit = token != 0 && c.cached && c.cachedToken == token && c.cachedStart == start
                     && c.cachedCount == count && c.device == device
                     && std::memcmp(&c.cachedWave, &wave, sizeof(wave)) == 0;
    MbsPackedBeams &packed = c.packed;
    mbs_po_beams view{};
    if (!hit)
    {
        std::string err;
        const int prc = mbs_pack_prepared(prepared, start, count, false, packed, &err);
        if (prc == MBS_PO_EBEAM)
            return false;   // reference: failDirect("bad-edge-data")
        if (prc != MBS_PO_OK)
            return false;
        view = packed.view(false);
        if (env_is("MBS_GPU_BEAM_STATS", "1"))
        {
            char line[1024];
            mbs_po_beam_stats(&view, line, (int)sizeof(line));
            std::fprintf(stderr, "%s\n", line);
        }
        if (view.n_beams == 0)
            return true;
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (!HandlerPOBoundary::Prepare(h, sphere, wave, device))
        return false;
    mbs_po_stats st;
    std::memset(&st, 0, sizeof(st));
    const auto t2 = std::chrono::steady_clock::now();
    int rc;
    if (token != 0)
    {
        if (!hit)
        {
            // (re)fill the cache: the staged beams stay on the device
            rc = c.cached ? mbs_po_restage(c.ctx, &view, c.cached) : mbs_po_stage(c.ctx, &view, &c.cached);
            if (rc != MBS_PO_OK)
            {
                c.cachedToken = 0;
                if (rc == MBS_PO_EBEAM)
                    return false;
                return report(rc, "staging");
            }
            c.cachedToken = token;
            c.cachedStart = start;
            c.cachedCount = count;
            c.cachedWave = wave;
        }
        rc = mbs_po_diffract_staged_pinned(c.ctx, c.cached, precision_from_env(), Mv,
                                           computeNoShadow ? Mnv : nullptr, &st);
    }
    else
    {
        rc = mbs_po_diffract_pinned(c.ctx, &view, precision_from_env(), Mv,
                                    computeNoShadow ? Mnv : nullptr, &st);
    }
    if (rc == MBS_PO_EBEAM)
        return false;
    if (!report(rc, "diffraction"))
        return false;
    if (timing)
    {
        const auto t3 = std::chrono::steady_clock::now();
        auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
            return std::chrono::duration<double, std::milli>(b - a).count();
        };
        double pr[6] = {};
        mbs_po_last_profile(c.ctx, pr, 6);
        std::fprintf(stderr,
                     "GPU timing diffract path=b200-%s device=%d orient=%d beams=%lld nAz=%d nZen=%d "
                     "cache=%s pack=%.3fms h2d+stage=%.3fms kernels=%.3fms reduce=%.3fms "
                     "total=%.3fms setup=%.3fms call=%.3fms "
                     "[grow=%.3f h2d=%.3f build=%.3f enqueue=%.3f wait=%.3f result=%.3f]\n",
                     precision_from_env() == MBS_PO_FP32C ? "fp32c" : "fp64", device, count,
                     hit ? -1LL : (long long)view.n_beams, nAz, nZen,
                     token == 0 ? "off" : (hit ? "hit" : "fill"), ms(t0, t1), st.h2d_ms,
                     st.kernel_ms, st.reduce_ms, ms(t0, t3), ms(t1, t2), ms(t2, t3),
                     pr[0], pr[1], pr[2], pr[3], pr[4], pr[5]);
    }
    return true;
}

// Persistent worker thread per device for the multi-device split.  Each keeps
// its own BoundaryContext (device context, grid, staged batches) from call to
// call, where the reference starts std::async threads per call
// (GpuDiffraction.cu:4214-4250).  Never destroyed: idle workers wait until
// the process exits.
class DeviceWorkers
{
public:
    static DeviceWorkers &get()
    {
        static DeviceWorkers *w = new DeviceWorkers();
        return *w;
    }

    // fns[d] on device d's worker, all at once; true when all succeeded
    bool run(const std::vector<std::function<bool()>> &fns)
    {
        while (workers_.size() < fns.size())
            workers_.emplace_back(new Worker((int)workers_.size()));
        for (size_t d = 0; d < fns.size(); ++d)
        {
            Worker &w = *workers_[d];
            std::lock_guard<std::mutex> lk(w.m);
            w.job = fns[d];
            w.has = true;
            w.done = false;
            w.cv.notify_all();
        }
        bool ok = true;
        for (size_t d = 0; d < fns.size(); ++d)
        {
            Worker &w = *workers_[d];
            std::unique_lock<std::mutex> lk(w.m);
            w.cv.wait(lk, [&] { return w.done; });
            ok = w.ok && ok;
        }
        return ok;
    }

private:
    struct Worker
    {
        std::mutex m;
        std::condition_variable cv;
        std::function<bool()> job;
        bool has = false, done = false, ok = false;
        std::thread th;
        explicit Worker(int device) : th(&Worker::loop, this, device) { th.detach(); }
        void loop(int device)
        {
            cudaSetDevice(device);
            g_multiWorker = true;
            for (;;)
            {
                std::function<bool()> f;
                {
                    std::unique_lock<std::mutex> lk(m);
                    cv.wait(lk, [&] { return has; });
                    f.swap(job);
                    has = false;
                }
                const bool r = f();
                std::lock_guard<std::mutex> lk(m);
                ok = r;
                done = true;
                cv.notify_all();
            }
        }
    };
    std::vector<std::unique_ptr<Worker>> workers_;
};

static bool diffract_range(HandlerPO &h, const ScatteringRange &sphere,
                           const std::vector<PreparedOrientation> &prepared,
                           int start, int count, Arr2D &localM,
                           Arr2D &localM_noshadow, bool computeNoShadow, int device)
{
    const int nAz = sphere.nAzimuth, nZen = sphere.nZenith;
    const int nDev = g_multiWorker ? 1 : multi_devices(count);
    if (nDev > 1)
    {
        // contiguous ranges, one per device, summed into localM in device
        // order (GpuDiffraction.cu:4185-4270)
        static bool printed = false;
        if (!printed || env_is("MBS_GPU_MULTI_DEBUG", "1"))
        {
            std::fprintf(stderr,
                         "GPU multi-device: using %d visible CUDA devices for %d orientations in this batch "
                         "(disable with MBS_GPU_MULTI=0, cap with MBS_GPU_MULTI_MAX=N).\n",
                         nDev, count);
            printed = true;
        }
        std::vector<const double *> pm(nDev, nullptr), pn(nDev, nullptr);
        std::vector<std::function<bool()>> jobs;
        for (int dev = 0; dev < nDev; ++dev)
        {
            int begin = 0, sub = 0;
            mbs_po_device_range(start, count, nDev, dev, &begin, &sub);
            jobs.push_back([&h, &sphere, &prepared, &pm, &pn, begin, sub, computeNoShadow, dev]() {
                if (sub <= 0)
                    return true;
                return diffract_core(h, sphere, prepared, begin, sub, computeNoShadow, dev, &pm[dev],
                                     &pn[dev]);
            });
        }
        if (!DeviceWorkers::get().run(jobs))
            return false;
        for (int dev = 0; dev < nDev; ++dev)
        {
            if (pm[dev])
                add_plane(pm[dev], localM, nAz, nZen + 1);
            if (pn[dev])
                add_plane(pn[dev], localM_noshadow, nAz, nZen + 1);
        }
        return true;
    }
    const bool timing = env_is("MBS_GPU_TIMING", "1");
    const auto t0 = std::chrono::steady_clock::now();
    const double *Mv = nullptr, *Mnv = nullptr;
    if (!diffract_core(h, sphere, prepared, start, count, computeNoShadow, device, &Mv, &Mnv))
        return false;
    const auto t1 = std::chrono::steady_clock::now();
    if (Mv)
        add_plane(Mv, localM, nAz, nZen + 1);
    if (Mnv)
        add_plane(Mnv, localM_noshadow, nAz, nZen + 1);
    if (timing && Mv)
        std::fprintf(stderr, "GPU timing add path=b200 call=%.3fms add=%.3fms\n",
                     std::chrono::duration<double, std::milli>(t1 - t0).count(),
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count());
    return true;
}

// Size-scaled diffraction of prepared[start, start+count) at every factor of
// `scales` in one call (mbs_po_diffract_multisize): Mueller sums added into
// *Ms[i], the no-shadow sums into *Mns[i] when Mns is given.
static bool diffract_scaled(HandlerPO &h, const ScatteringRange &sphere,
                            const std::vector<PreparedOrientation> &prepared, int start,
                            int count, const std::vector<double> &scales, double waveIndex,
                            const std::vector<Arr2D *> &Ms, const std::vector<Arr2D *> *Mns,
                            int device)
{
    const int nAz = sphere.nAzimuth, nZen = sphere.nZenith;
    MbsPackedBeams packed;
    std::string err;
    const int prc = mbs_pack_prepared(prepared, start, count, true, packed, &err);
    if (prc != MBS_PO_OK)
        return false;   // reference: failMultiK("bad-edge-data")
    const mbs_po_beams view = packed.view(true);
    if (view.n_beams == 0)
        return true;
    if (!HandlerPOBoundary::Prepare(h, sphere, HandlerPOWaveAccess::Get(h, 0.0), device))
        return false;
    BoundaryContext &c = g_ctx;
    const size_t plane = (size_t)nAz * (nZen + 1) * 16;
    const size_t n = plane * scales.size();
    c.M.assign(n, 0.0);
    if (Mns)
        c.Mns.assign(n, 0.0);
    mbs_po_stats st;
    std::memset(&st, 0, sizeof(st));
    const int rc = mbs_po_diffract_multisize(c.ctx, &view, scales.data(), (int)scales.size(),
                                             waveIndex, precision_from_env(), c.M.data(),
                                             Mns ? c.Mns.data() : nullptr, &st);
    if (rc == MBS_PO_EBEAM)
        return false;
    if (!report(rc, "multi-size diffraction"))
        return false;
    for (size_t s = 0; s < scales.size(); ++s)
    {
        add_plane(c.M.data() + s * plane, *Ms[s], nAz, nZen + 1);
        if (Mns)
            add_plane(c.Mns.data() + s * plane, *(*Mns)[s], nAz, nZen + 1);
    }
    if (env_is("MBS_GPU_TIMING", "1"))
        std::fprintf(stderr,
                     "GPU timing multik path=b200-%s orient=%d sizes=%zu beams=%lld nAz=%d nZen=%d "
                     "h2d+stage=%.3fms kernels=%.3fms reduce=%.3fms\n",
                     precision_from_env() == MBS_PO_FP32C ? "fp32c" : "fp64", view.n_orient,
                     scales.size(), (long long)view.n_beams, nAz, nZen, st.h2d_ms, st.kernel_ms,
                     st.reduce_ms);
    return true;
}

bool HandlerPO::HandleOrientationsToLocalGpu(const std::vector<PreparedOrientation> &prepared,
                                             int start, int count, Arr2D &localM,
                                             Arr2D &localM_noshadow, double scale,
                                             double waveIndex)
{
    if (!isCoh)
        return false;
    if (start < 0 || count < 0 || start > (int)prepared.size())
        return false;
    if (std::fabs(scale - 1.0) > 1e-15)
    {
        // scaled packing (GpuDiffraction.cu:4323-4324): one size instance
        const std::vector<double> scales(1, scale);
        const std::vector<Arr2D *> Ms(1, &localM), Mns(1, &localM_noshadow);
        return diffract_scaled(*this, m_sphere, prepared, start, count, scales,
                               waveIndex > 0.0 ? waveIndex : 0.0, Ms,
                               ComputeNoShadow() ? &Mns : nullptr, current_device());
    }
    return diffract_range(*this, m_sphere, prepared, start, count, localM, localM_noshadow,
                          ComputeNoShadow(), current_device());
}

bool HandlerPO::HandleOrientationsToLocalGpu(const std::vector<PreparedOrientation> &prepared,
                                             Arr2D &localM, Arr2D &localM_noshadow)
{
    return HandleOrientationsToLocalGpu(prepared, 0, (int)prepared.size(), localM,
                                        localM_noshadow, 1.0, 0.0);
}

bool HandlerPO::HandleOrientationsToLocalGpuOnDevice(
    const std::vector<PreparedOrientation> &prepared, int start, int count, int device,
    Arr2D &localM, Arr2D &localM_noshadow, double scale, double waveIndex,
    unsigned long long cacheToken)
{
    // the call stays on `device` (no further split) and reuses the staged
    // beams of an earlier call with the same token and range
    // (GpuDiffraction.cu:3464-3500)
    int saved = 0;
    cudaGetDevice(&saved);
    if (cudaSetDevice(device) != cudaSuccess)
        return false;
    const bool prevWorker = g_multiWorker;
    const unsigned long long prevToken = g_cacheToken;
    g_multiWorker = true;
    g_cacheToken = std::fabs(scale - 1.0) > 1e-15 ? 0 : cacheToken;   // scaled calls: no cache
    const bool ok = HandleOrientationsToLocalGpu(prepared, start, count, localM,
                                                 localM_noshadow, scale, waveIndex);
    g_multiWorker = prevWorker;
    g_cacheToken = prevToken;
    cudaSetDevice(saved);
    return ok;
}

bool HandlerPO::HandleBeamsToLocalGpu(const PreparedOrientation &prepared, Arr2D &localM,
                                      Arr2D &localM_noshadow)
{
    std::vector<PreparedOrientation> one(1, prepared);
    return HandleOrientationsToLocalGpu(one, 0, 1, localM, localM_noshadow, 1.0, 0.0);
}

namespace
{

// MBS_FFT_PHI_FACTOR: 1..64, or "auto"/unset (0), as the reference reads it
// (GpuDiffraction.cu:514-530).
int fft_phi_factor_env()
{
    const char *v = std::getenv("MBS_FFT_PHI_FACTOR");
    if (!v || !*v)
        return 0;
    char *end = nullptr;
    const long f = std::strtol(v, &end, 10);
    if (!end || *end != '\0' || f < 1 || f > 64)
        return 0;
    return (int)f;
}

// Azimuth factor of the FFT-phi path (choose_fft_phi_factor,
// GpuDiffraction.cu:712-726): the handler's configured factor, else the
// environment's, else by the output azimuth count.
int fft_phi_factor(int nFull, int configured)
{
    if (configured > 0)
        return configured;
    const int env = fft_phi_factor_env();
    if (env > 0)
        return env;
    if (nFull >= 2400)
        return 8;
    if (nFull >= 600)
        return 6;
    if (nFull >= 240)
        return 3;
    return 2;
}

// The interpolated grid against the one from twice the direct azimuths
// (report_fft_check, GpuDiffraction.cu:3142-3204): the larger of the maximum
// relative M11 error over directions with M11 >= 1e-3 of the grid's maximum,
// and of the maximum error of any element relative to max(|M11|, that floor).
double fft_check_estimate(const std::vector<double> &fft, const std::vector<double> &ref,
                          int nAz, int nRows, const char *name)
{
    double refMax = 0.0;
    for (int i = 0; i < nAz * nRows; ++i)
        refMax = std::max(refMax, std::fabs(ref[(size_t)i * 16]));
    const double significant = 1e-3 * refMax;
    double sigRel = 0.0, normRel = 0.0, maxRel = 0.0;
    for (int i = 0; i < nAz * nRows; ++i) {
        const double a = ref[(size_t)i * 16], b = fft[(size_t)i * 16];
        const double rel = std::fabs(b - a) / std::max(std::fabs(a), 1e-12);
        maxRel = std::max(maxRel, rel);
        if (std::fabs(a) >= significant)
            sigRel = std::max(sigRel, rel);
        const double scale = std::max(std::fabs(a), significant);
        for (int e = 0; e < 16; ++e)
            normRel = std::max(normRel, std::fabs(fft[(size_t)i * 16 + e] - ref[(size_t)i * 16 + e]) / scale);
    }
    std::fprintf(stderr, "GPU FFT check %s: M11 max_rel=%.6g significant_max_rel=%.6g "
                 "Mueller/M11 max_rel=%.6g\n", name, maxRel, sigRel, normRel);
    return std::max(sigRel, normRel);
}

}  // namespace

// Direct evaluation of prepared[start, start+count) on `low` (n_az azimuth
// bins), interpolated on the device to nFull bins: adds into M (and Mns),
// flat [nFull][nZen+1][16].
static bool diffract_fft_phi(HandlerPO &h, const ScatteringRange &low,
                             const std::vector<PreparedOrientation> &prepared, int start, int count,
                             int nFull, std::vector<double> &M, std::vector<double> *Mns, int device)
{
    const bool timing = env_is("MBS_GPU_TIMING", "1");
    const auto t0 = std::chrono::steady_clock::now();
    MbsPackedBeams packed;
    std::string err;
    const int prc = mbs_pack_prepared(prepared, start, count, false, packed, &err);
    if (prc != MBS_PO_OK)
        return false;
    const mbs_po_beams view = packed.view(false);
    if (view.n_beams == 0)
        return true;
    if (!HandlerPOBoundary::Prepare(h, low, HandlerPOWaveAccess::Get(h, 0.0), device))
        return false;
    mbs_po_stats st;
    std::memset(&st, 0, sizeof(st));
    const int rc = mbs_po_diffract_fft_phi(g_ctx.ctx, &view, precision_from_env(), nFull, M.data(),
                                           Mns ? Mns->data() : nullptr, &st);
    if (rc == MBS_PO_EBEAM)
        return false;
    if (!report(rc, "FFT-phi diffraction"))
        return false;
    if (timing)
        std::fprintf(stderr,
                     "GPU timing fft_phi path=b200-%s orient=%d beams=%lld nPhiDirect=%d nPhiOut=%d "
                     "kernels=%.3fms total=%.3fms\n",
                     precision_from_env() == MBS_PO_FP32C ? "fp32c" : "fp64", view.n_orient,
                     (long long)view.n_beams, low.nAzimuth, nFull, st.kernel_ms,
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    return true;
}

bool HandlerPO::HandleOrientationsToLocalGpuFftPhi(const std::vector<PreparedOrientation> &prepared,
                                                   int start, int count, Arr2D &localM,
                                                   Arr2D &localM_noshadow, double scale,
                                                   double waveIndex)
{
    // Direct evaluation on nFull / factor azimuth bins, then the azimuth
    // interpolation of the reference's FFT-phi path on the device
    // (GpuDiffraction.cu:3504-3760): an approximation of the direct result on
    // the requested grid.  Not carried over: the environment-driven zenith
    // factor (MBS_FFT_THETA_FACTOR) and adaptive spike rows
    // (MBS_FFT_ADAPTIVE_PHI), both off by default there; size-scaled calls
    // take the direct path.
    if (!isCoh)
        return false;
    if (start < 0 || count < 0 || start > (int)prepared.size())
        return false;
    const int nFull = m_sphere.nAzimuth;
    const int nZen = m_sphere.nZenith;
    const int nRows = nZen + 1;
    const bool ns = ComputeNoShadow();
    const int factor = fft_phi_factor(nFull, m_fftPhiFactor);
    int nLow = factor > 1 ? nFull / factor : nFull;
    if (nLow < 16)
        nLow = std::min(nFull, 16);
    if (factor <= 1 || nFull < 32 || nLow >= nFull || std::fabs(scale - 1.0) > 1e-15)
    {
        if (m_fftStatistics)
            m_fftStatistics->RecordCall(nFull, nFull, 1);
        return HandleOrientationsToLocalGpu(prepared, start, count, localM, localM_noshadow,
                                            scale, waveIndex);
    }
    if (m_fftStatistics)
        m_fftStatistics->RecordCall(nFull, nLow, factor);
    static bool announced = false;
    if (!announced)
    {
        std::fprintf(stderr, "GPU FFT azimuth interpolation: direct Nphi=%d, output Nphi=%d "
                     "(factor=%d), on the B200 library\n", nLow, nFull, factor);
        announced = true;
    }
    auto sphere_with = [&](int nAz) {
        ScatteringRange s = m_sphere;
        s.nAzimuth = nAz;
        s.azinuthStep = M_2PI / nAz;
        s.ComputeSphereDirections(*m_incidentLight);
        return s;
    };
    const size_t n = (size_t)nFull * nRows * 16;
    std::vector<double> fftM(n, 0.0), fftMns(ns ? n : 0, 0.0);
    const int device = current_device();
    if (!diffract_fft_phi(*this, sphere_with(nLow), prepared, start, count, nFull, fftM,
                          ns ? &fftMns : nullptr, device))
        return false;
    const char *chk = std::getenv("MBS_FFT_CHECK");
    const bool doCheck = (chk && std::strcmp(chk, "1") == 0) || m_fftTolerance > 0.0;
    if (doCheck)
    {
        const int nCheck = std::min(nFull, 2 * nLow);
        std::vector<double> checkM(n, 0.0), checkMns(ns ? n : 0, 0.0);
        if (!diffract_fft_phi(*this, sphere_with(nCheck), prepared, start, count, nFull, checkM,
                              ns ? &checkMns : nullptr, device))
            return false;
        double est = fft_check_estimate(fftM, checkM, nFull, nRows, "full");
        if (ns)
            est = std::max(est, fft_check_estimate(fftMns, checkMns, nFull, nRows, "no-shadow"));
        const bool refine = m_fftTolerance > 0.0 && est > m_fftTolerance;
        if (m_fftStatistics)
            m_fftStatistics->RecordValidation(est, refine);
        if (refine)
        {
            fftM.swap(checkM);
            fftMns.swap(checkMns);
            std::fprintf(stderr, "GPU FFT validation exceeded tolerance: estimate=%.6g, "
                         "tolerance=%.6g; using the doubled direct Nphi=%d result\n",
                         est, m_fftTolerance, nCheck);
        }
    }
    add_plane(fftM.data(), localM, nFull, nRows);
    if (ns)
        add_plane(fftMns.data(), localM_noshadow, nFull, nRows);
    return true;
}

bool HandlerPO::HandleOrientationsToLocalGpuMultiK(const std::vector<PreparedOrientation> &prepared,
                                                   int start, int count,
                                                   const std::vector<double> &scales,
                                                   double waveIndex,
                                                   std::vector<Arr2D> &localMs)
{
    // Same refusals as the reference (GpuDiffraction.cu:3970-3975); the fused
    // path is on by default here, MBS_GPU_MULTI_K_FULL=0 turns it off so the
    // caller falls back to per-size calls.
    if (env_is("MBS_GPU_MULTI_K_FULL", "0"))
        return false;
    if (!isCoh || ComputeNoShadow())
        return false;
    if (count <= 0 || scales.empty())
        return true;
    if (localMs.size() < scales.size() || start < 0 || start > (int)prepared.size())
        return false;
    std::vector<Arr2D *> Ms;
    for (size_t s = 0; s < scales.size(); ++s)
        Ms.push_back(&localMs[s]);
    return diffract_scaled(*this, m_sphere, prepared, start, count, scales, waveIndex, Ms,
                           nullptr, current_device());
}

bool HandlerPO::HandleOrientationsToLocalGpuFftPhiMultiK(
    const std::vector<PreparedOrientation> &prepared, int start, int count,
    const std::vector<double> &scales, double waveIndex, std::vector<Arr2D> &localMs)
{
    return HandleOrientationsToLocalGpuMultiK(prepared, start, count, scales, waveIndex, localMs);
}

bool HandlerPO::DiffractThetasGpu(const std::vector<PreparedOrientation> &prepared,
                                  const double *theta_rads, int nPoints,
                                  std::vector<double> &m11_out)
{
    if (nPoints <= 0)
        return true;
    if (prepared.empty() || m_sphere.nAzimuth <= 0)
        return true;
    MbsPackedBeams packed;
    if (mbs_pack_prepared(prepared, 0, (int)prepared.size(), false, packed, nullptr) != MBS_PO_OK)
        return false;
    m11_out.assign(nPoints, 0.0);
    const mbs_po_beams view = packed.view(false);
    if (view.n_beams == 0)
        return true;
    if (!HandlerPOBoundary::Prepare(*this, m_sphere, HandlerPOWaveAccess::Get(*this, 0.0),
                                    current_device()))
        return false;
    const int rc = mbs_po_diffract_thetas(g_ctx.ctx, &view, theta_rads, nPoints, m11_out.data());
    if (rc == MBS_PO_EBEAM)
        return false;
    return report(rc, "theta scan");
}

int HandlerPO::SelectGpuOrientationBatchSize(const std::vector<PreparedOrientation> &prepared,
                                             int start, int maxCount) const
{
    if (maxCount <= 1)
        return std::max(1, maxCount);
    if (start < 0 || start > (int)prepared.size())
        return std::max(1, maxCount);
    // the selector reads only the orientations' beam and vertex counts: build
    // those, not the whole packed batch; a beam without valid edge data keeps
    // the full count, as a failed packing did
    const int n = std::min(maxCount, (int)prepared.size() - start);
    std::vector<int64_t> bo(n + 1, 0), vo(1, 0);
    for (int oi = 0; oi < n; ++oi)
    {
        for (const PreparedBeam &pb : prepared[start + oi].beams)
        {
            const int nv = pb.edgeData.nVertices;
            if (!pb.edgeData.valid || nv < 3 || nv >= BeamEdgeData::MAX_EDGES)
                return std::max(1, maxCount);
            vo.push_back(vo.back() + nv);
        }
        bo[oi + 1] = (int64_t)vo.size() - 1;
    }
    if (!HandlerPOBoundary::Prepare(*this, m_sphere, HandlerPOWaveAccess::Get(*this, 0.0),
                                    current_device()))
        return std::max(1, maxCount);
    mbs_po_beams view{};
    view.n_orient = n;
    view.n_beams = bo[n];
    view.n_verts = vo.back();
    view.beam_offsets = bo.data();
    view.vert_offsets = vo.data();
    int count = maxCount;
    if (mbs_po_select_batch(g_ctx.ctx, &view, 0, maxCount, mem_fraction(), &count) != MBS_PO_OK)
        return std::max(1, maxCount);
    int selected = std::max(1, count);
    if (!g_multiWorker)
    {
        // the batch is split over the devices (GpuDiffraction.cu:3021-3027)
        const int nDev = multi_devices(maxCount);
        if (nDev > 1)
            selected = std::min(maxCount, selected * nDev);
    }
    return selected;
}
