// producer.cpp — the reference's host beam producer behind a C ABI
// (include/mbs_host.h).
//
// Builds the same particle, light, scattering and HandlerPO objects as the
// reference CLI (reference src/main.cpp:1655-1760 particle, :2228-2252 tracer
// and handler, :196-260 cutoff profiles) and runs phase 1 of
// TracerPOTotal::TraceWeightedOrientations (TracerPOTotal.cpp:5815-5898):
// per OpenMP thread a private Particle / Scattering / HandlerPO, then for each
// orientation Rotate -> FormShadowBeam -> ScatterLight -> PrepareBeams.  The
// prepared orientations are flattened with mbs_pack_prepared.
#include "mbs_host.h"
#include "beam_pack.h"
#include "prepare.h"

#include "HandlerPOTotal.h"
#include "Hexagonal.h"
#include "Bullet.h"
#include "Droxtal.h"
#include "ConcaveHexagonal.h"
#include "HexagonalAggregate.h"
#include "TracerPOTotal.h"
#include "Sobol.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

struct mbs_host_batch
{
    MbsPackedBeams packed;
    mbs_po_beams view;
    double trace_seconds = 0.0;
    // thread-summed seconds in ScatterLight (with the shadow beam) and in
    // PrepareBeams, and seconds of packing into the flat batch (the
    // per-orientation appends summed over threads plus the final gather)
    double phase_seconds[3] = {0.0, 0.0, 0.0};
};

namespace
{

void set_err(char *err, int errlen, const std::string &msg)
{
    if (err && errlen > 0)
    {
        std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
    }
}

// Exposes the protected wave constants of Handler.
class HostHandlerPO : public HandlerPOTotal
{
public:
    using HandlerPOTotal::HandlerPOTotal;
    void FillWave(mbs_po_wave &w) const
    {
        w.wave_index = m_waveIndex;
        w.wavelength = m_wavelength;
        w.compl_wave_re = real(m_complWave);
        w.compl_wave_im = imag(m_complWave);
        w.inv_compl_wave_re = real(m_invComplWave);
        w.inv_compl_wave_im = imag(m_invComplWave);
        w.eps1 = m_eps1;
        w.abs_coeff = m_cAbs;
        w.ot_far_reference_path = m_otFarReferencePath;
        w.ot_ping_distance = m_otPingDistance;
        w.legacy_sign = m_legacySign ? 1 : 0;
        w.ot_phase_average = m_otPhaseAverage ? 1 : 0;
    }
};

// Reference objects for one configuration (mirrors src/main.cpp).
struct HostSetup
{
    std::unique_ptr<Particle> particle;
    std::unique_ptr<TracerPOTotal> tracer;
    std::unique_ptr<HostHandlerPO> handler;
    Tracks tracks;
    bool isAbs = false;

    explicit HostSetup(const mbs_host_config &cfg)
    {
        isAbs = cfg.absorption != 0 || cfg.ri_im != 0.0;
        const ::complex ri(cfg.ri_re, isAbs ? cfg.ri_im : 0.0);
        if (cfg.particle_file && cfg.particle_file[0])
        {
            particle.reset(new Particle());
            particle->SetFromFile(cfg.particle_file);
            particle->SetRefractiveIndex(ri);
            if (cfg.resize > 0.0)
                particle->Resize(cfg.resize);
        }
        else
        {
            switch (cfg.particle_type)
            {
            case 1:   // --particle 1 L D  (main.cpp:1731-1735)
                particle.reset(new Hexagonal(ri, cfg.p[1], cfg.p[0]));
                break;
            case 2:   // --particle 2 L D  (main.cpp:1736-1741)
            {
                const double sup = (cfg.p[1] * std::sqrt(3) * std::tan(DegToRad(62))) / 4;
                particle.reset(new Bullet(ri, cfg.p[1], cfg.p[0], sup));
                break;
            }
            case 4:   // --particle 4 size  (main.cpp:1750-1755)
                particle.reset(new Droxtal(ri, DegToRad(32.35), DegToRad(71.81), cfg.p[0]));
                break;
            case 10:  // --particle 10 L D depth  (main.cpp:1762-1768)
                particle.reset(new ConcaveHexagonal(ri, cfg.p[1], cfg.p[0], cfg.p[2]));
                break;
            case 12:  // --particle 12 L D n  (main.cpp:1769-1775)
                particle.reset(new HexagonalAggregate(ri, cfg.p[1], cfg.p[0], (int)cfg.p[2]));
                break;
            default:
                throw std::invalid_argument("unsupported particle type " + std::to_string(cfg.particle_type));
            }
        }
        tracer.reset(new TracerPOTotal(particle.get(), cfg.max_reflections, "mbs_b200_host"));
        tracer->m_scattering->m_wave = cfg.wavelength;
        Scattering *sc = tracer->m_scattering;
        const int profile = cfg.cutoff_profile;
        if (profile < 0 || profile > 4)
            throw std::invalid_argument("unknown cutoff profile " + std::to_string(profile));
        if (profile == 1)
        {   // --cutoff-profile off (main.cpp:190-196)
            sc->restriction = std::numeric_limits<double>::infinity();
            sc->m_traceCutoffJRel = 0.0;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = 0.0;
        }
        else if (profile == 0)
        {   // legacy-default profile (main.cpp:197-206)
            sc->m_traceCutoffJRel = 1e-7;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = 0.0;
        }
        else
        {   // safe / balanced / fast (main.cpp:207-215)
            sc->m_traceCutoffJRel = 0.0;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = profile == 2 ? 1e-12 : (profile == 3 ? 1e-10 : 1e-8);
            sc->restriction = profile == 2 ? 1e8 : (profile == 3 ? 1e5 : 1e3);
        }
        tracer->shadowOff = cfg.shadow_off != 0;
        handler.reset(new HostHandlerPO(particle.get(), &tracer->m_incidentLight,
                                        1, cfg.wavelength));
        handler->isCoh = true;
        handler->m_legacySign = cfg.legacy_sign != 0;
        if (profile == 1)
        {   // main.cpp:131-137
            handler->m_targetEps = 0.0;
            handler->m_beamCutoffJRel = 0.0;
            handler->m_beamCutoffAreaRel = 0.0;
            handler->m_beamCutoffImportanceRel = 0.0;
        }
        else if (profile >= 2)
        {   // main.cpp:138-145
            handler->m_targetEps = 0.0;
            handler->m_beamCutoffJRel = 0.0;
            handler->m_beamCutoffAreaRel = 0.0;
            handler->m_beamCutoffImportanceRel = profile == 2 ? 1e-10 : (profile == 3 ? 1e-8 : 1e-6);
        }
        // individual thresholds after the profile, as the CLI applies them
        if (cfg.trace_cutoff_importance > 0.0)
            sc->m_traceCutoffImportanceRel = cfg.trace_cutoff_importance;
        if (cfg.beam_cutoff_importance > 0.0)
            handler->m_beamCutoffImportanceRel = cfg.beam_cutoff_importance;
        // PrepareBeams does not read the scattering grid; a 1x1 placeholder
        // keeps the per-track matrices of SetTracks small.
        handler->SetScatteringSphere(ScatteringRange(0, M_PI, 1, 1));
        handler->SetTracks(&tracks);
        handler->SetAbsorptionAccounting(isAbs);
        tracer->SetHandler(handler.get());
    }
};

}  // namespace

extern "C" int mbs_host_trace(const mbs_host_config *cfg, int n_orient,
                              const double *beta, const double *gamma,
                              const double *alpha, const double *weight,
                              mbs_host_batch **out, char *err, int errlen)
{
    if (!cfg || !out || n_orient < 0 || (n_orient > 0 && (!beta || !gamma || !weight)))
    {
        set_err(err, errlen, "mbs_host_trace: bad arguments");
        return MBS_PO_EINVAL;
    }
    *out = nullptr;
    try
    {
        HostSetup setup(*cfg);
        const auto t0 = std::chrono::steady_clock::now();
        Scattering *master = setup.tracer->m_scattering;
        master->PrepareForParallelTrace();
        bool failed = false;
        int failCode = MBS_PO_EINVAL;
        std::string failMsg;
        double scatterSeconds = 0.0, prepareSeconds = 0.0, packSeconds = 0.0;
        const int nThreads = cfg->n_threads > 0 ? cfg->n_threads : omp_get_max_threads();
        // Every worker prepares into one reused PreparedOrientation and
        // appends its flat records to its own part; the parts are gathered
        // in orientation order at the end.  (A PreparedBeam is about 5 KB;
        // materialising all of them at once costs more in first-touch page
        // faults than preparing them.)
        struct Slice
        {
            int part = 0;
            int64_t b0 = 0, nb = 0, v0 = 0, nv = 0, a0 = 0, na = 0;
            double ext = 0.0;
        };
        std::vector<Slice> slices(n_orient);
        std::vector<MbsPackedBeams> parts(nThreads);
#pragma omp parallel num_threads(nThreads)
        {
            const int tid = omp_get_thread_num();
            MbsPackedBeams &part = parts[tid];
            Particle localParticle = *setup.particle;
            Scattering *localScatter = master->CloneFor(&localParticle, &setup.tracer->m_incidentLight);
            PrepareHandler localHandler(&localParticle, &setup.tracer->m_incidentLight,
                                        setup.handler->nTheta, master->m_wave);
            const bool referencePrepare = cfg->reference_prepare != 0;
            localHandler.ConfigureForThreadLocalPrepare(*setup.handler, localScatter);
            // the producer packs the prepared beams: only what the batch reads
            localHandler.SetBatchOnly(true);
            std::vector<Beam> localBeams;
            PreparedOrientation po;
            double tScatter = 0.0, tPrepare = 0.0, tPack = 0.0;
#pragma omp for schedule(dynamic, 1)
            for (int i = 0; i < n_orient; ++i)
            {
                try
                {
                    const auto a = std::chrono::steady_clock::now();
                    localParticle.Rotate(beta[i], gamma[i], alpha ? alpha[i] : 0.0);
                    if (!setup.tracer->shadowOff)
                        localScatter->FormShadowBeam(localBeams);
                    const bool ok = localScatter->ScatterLight(0, 0, localBeams);
                    const auto b = std::chrono::steady_clock::now();
                    if (ok && referencePrepare)
                        localHandler.PrepareBeams(localBeams, weight[i], po);
                    else if (ok)
                        localHandler.Prepare(localBeams, weight[i], po);
                    else
                    {
                        po.beams.clear();
                        po.sinZenith = weight[i];
                        po.extinctionOt = 0.0;
                    }
                    localBeams.clear();
                    const auto c = std::chrono::steady_clock::now();
                    Slice &sl = slices[i];
                    sl.part = tid;
                    sl.b0 = (int64_t)part.beam_flags.size();
                    sl.v0 = (int64_t)part.vx.size();
                    sl.a0 = (int64_t)part.abs_paths.size();
                    std::string perr;
                    const int prc = mbs_pack_append(po, true, part, &perr);
                    if (prc != MBS_PO_OK)
                    {
#pragma omp critical(mbs_host_trace_err)
                        {
                            failed = true;
                            failCode = prc;
                            failMsg = perr;
                        }
                    }
                    sl.nb = (int64_t)part.beam_flags.size() - sl.b0;
                    sl.nv = (int64_t)part.vx.size() - sl.v0;
                    sl.na = (int64_t)part.abs_paths.size() - sl.a0;
                    sl.ext = po.extinctionOt;
                    tScatter += std::chrono::duration<double>(b - a).count();
                    tPrepare += std::chrono::duration<double>(c - b).count();
                    tPack += std::chrono::duration<double>(std::chrono::steady_clock::now() - c).count();
                }
                catch (const std::exception &e)
                {
#pragma omp critical(mbs_host_trace_err)
                    {
                        failed = true;
                        failMsg = "tracing failed: " + std::string(e.what());
                    }
                }
            }
            delete localScatter;
#pragma omp critical(mbs_host_trace_time)
            {
                scatterSeconds += tScatter;
                prepareSeconds += tPrepare;
                packSeconds += tPack;
            }
        }
        if (failed)
        {
            set_err(err, errlen, failMsg);
            return failCode;
        }
        // gather the parts in orientation order
        const auto tg = std::chrono::steady_clock::now();
        std::unique_ptr<mbs_host_batch> batch(new mbs_host_batch());
        MbsPackedBeams &pk = batch->packed;
        std::vector<int64_t> B0(n_orient + 1, 0), V0(n_orient + 1, 0), A0(n_orient + 1, 0);
        for (int i = 0; i < n_orient; ++i)
        {
            B0[i + 1] = B0[i] + slices[i].nb;
            V0[i + 1] = V0[i] + slices[i].nv;
            A0[i + 1] = A0[i] + slices[i].na;
        }
        const int64_t nB = B0[n_orient], nV = V0[n_orient], nA = A0[n_orient];
        pk.beam_offsets.assign(n_orient + 1, 0);
        pk.orient_weight.assign(n_orient, 0.0);
        pk.extinction_ot.assign(n_orient, 0.0);
        pk.vert_offsets.resize(nB + 1);
        pk.vx.resize(nV);
        pk.vy.resize(nV);
        pk.slope_yx.resize(nV);
        pk.slope_xy.resize(nV);
        pk.edge_flags.resize(nV);
        pk.beam_geom.resize((size_t)nB * MBS_PO_GEOM_STRIDE);
        pk.beam_flags.resize(nB);
        pk.beam_raw.resize((size_t)nB * MBS_PO_RAW_STRIDE);
        pk.abs_offsets.resize(nB + 1);
        pk.abs_paths.resize(nA);
        pk.max_vertices = 0;
        for (const MbsPackedBeams &pt : parts)
            pk.max_vertices = std::max(pk.max_vertices, pt.max_vertices);
#pragma omp parallel for schedule(dynamic, 16) num_threads(nThreads)
        for (int i = 0; i < n_orient; ++i)
        {
            const Slice &sl = slices[i];
            const MbsPackedBeams &pt = parts[sl.part];
            pk.beam_offsets[i] = B0[i];
            pk.orient_weight[i] = weight[i];
            pk.extinction_ot[i] = sl.ext;
            for (int64_t k = 0; k < sl.nb; ++k)
            {
                pk.vert_offsets[B0[i] + k] = pt.vert_offsets[sl.b0 + k] - sl.v0 + V0[i];
                pk.abs_offsets[B0[i] + k] = pt.abs_offsets[sl.b0 + k] - sl.a0 + A0[i];
            }
            std::copy_n(pt.vx.begin() + sl.v0, sl.nv, pk.vx.begin() + V0[i]);
            std::copy_n(pt.vy.begin() + sl.v0, sl.nv, pk.vy.begin() + V0[i]);
            std::copy_n(pt.slope_yx.begin() + sl.v0, sl.nv, pk.slope_yx.begin() + V0[i]);
            std::copy_n(pt.slope_xy.begin() + sl.v0, sl.nv, pk.slope_xy.begin() + V0[i]);
            std::copy_n(pt.edge_flags.begin() + sl.v0, sl.nv, pk.edge_flags.begin() + V0[i]);
            std::copy_n(pt.beam_geom.begin() + sl.b0 * MBS_PO_GEOM_STRIDE, sl.nb * MBS_PO_GEOM_STRIDE,
                        pk.beam_geom.begin() + B0[i] * MBS_PO_GEOM_STRIDE);
            std::copy_n(pt.beam_flags.begin() + sl.b0, sl.nb, pk.beam_flags.begin() + B0[i]);
            std::copy_n(pt.beam_raw.begin() + sl.b0 * MBS_PO_RAW_STRIDE, sl.nb * MBS_PO_RAW_STRIDE,
                        pk.beam_raw.begin() + B0[i] * MBS_PO_RAW_STRIDE);
            std::copy_n(pt.abs_paths.begin() + sl.a0, sl.na, pk.abs_paths.begin() + A0[i]);
        }
        pk.beam_offsets[n_orient] = nB;
        pk.vert_offsets[nB] = nV;
        pk.abs_offsets[nB] = nA;
        batch->phase_seconds[0] = scatterSeconds;
        batch->phase_seconds[1] = prepareSeconds;
        batch->phase_seconds[2] = packSeconds
            + std::chrono::duration<double>(std::chrono::steady_clock::now() - tg).count();
        batch->view = batch->packed.view(true);
        batch->trace_seconds = std::chrono::duration<double>(
            std::chrono::steady_clock::now() - t0).count();
        *out = batch.release();
        return MBS_PO_OK;
    }
    catch (const std::exception &e)
    {
        set_err(err, errlen, std::string("mbs_host_trace: ") + e.what());
        return MBS_PO_EINVAL;
    }
}

extern "C" const mbs_po_beams *mbs_host_batch_view(const mbs_host_batch *batch)
{
    return batch ? &batch->view : nullptr;
}

extern "C" double mbs_host_batch_extinction(const mbs_host_batch *batch, int o)
{
    if (!batch || o < 0 || o >= (int)batch->packed.extinction_ot.size())
        return 0.0;
    return batch->packed.extinction_ot[o];
}

extern "C" int mbs_host_batch_phase_seconds(const mbs_host_batch *batch, double *out3)
{
    if (!batch || !out3)
        return MBS_PO_EINVAL;
    for (int i = 0; i < 3; ++i)
        out3[i] = batch->phase_seconds[i];
    return MBS_PO_OK;
}

extern "C" double mbs_host_batch_trace_seconds(const mbs_host_batch *batch)
{
    return batch ? batch->trace_seconds : 0.0;
}

extern "C" void mbs_host_batch_free(mbs_host_batch *batch)
{
    delete batch;
}

extern "C" int mbs_host_symmetry(const mbs_host_config *cfg, double *beta_sym,
                                 double *gamma_sym, double *dmax)
{
    if (!cfg)
        return MBS_PO_EINVAL;
    try
    {
        HostSetup setup(*cfg);
        const Symmetry &s = setup.particle->GetSymmetry();
        if (beta_sym) *beta_sym = s.beta;
        if (gamma_sym) *gamma_sym = s.gamma;
        if (dmax) *dmax = setup.particle->MaximalDimention();
        return MBS_PO_OK;
    }
    catch (...)
    {
        return MBS_PO_EINVAL;
    }
}

extern "C" int mbs_host_sobol_orientations(int n, unsigned seed, double beta_sym,
                                           double gamma_sym, double *beta,
                                           double *gamma, double *weight)
{
    if (n <= 0 || !beta || !gamma || !weight)
        return MBS_PO_EINVAL;
    // TracerPOTotal::TraceFromSobolSeed (TracerPOTotal.cpp:5476-5488).
    Sobol2D sobol(seed);
    std::vector<double> su, sv;
    sobol.generate(n, su, sv);
    const double cosBetaSym = std::cos(beta_sym);
    const double w = 1.0 / n;
    for (int i = 0; i < n; ++i)
    {
        beta[i] = std::acos(1.0 - (1.0 - cosBetaSym) * su[i]);
        gamma[i] = gamma_sym * sv[i];
        weight[i] = w;
    }
    return MBS_PO_OK;
}

extern "C" int mbs_host_wave(const mbs_host_config *cfg, mbs_po_wave *wave)
{
    if (!cfg || !wave)
        return MBS_PO_EINVAL;
    try
    {
        HostSetup setup(*cfg);
        std::memset(wave, 0, sizeof(*wave));
        setup.handler->FillWave(*wave);
        return MBS_PO_OK;
    }
    catch (...)
    {
        return MBS_PO_EINVAL;
    }
}

extern "C" int mbs_host_grid(double zen_start_deg, double zen_end_deg, int n_az,
                             int n_zen, const double *theta_deg, double *theta,
                             double *vf, double *dcos2pi, double *az_step)
{
    if (n_az <= 0 || n_zen <= 0 || !theta || !vf)
        return MBS_PO_EINVAL;
    ScatteringRange range(DegToRad(zen_start_deg), DegToRad(zen_end_deg), n_az, n_zen);
    if (theta_deg)
    {
        // LoadThetaGrid without a file (Handler.h:31-61).
        range.thetaValues.clear();
        for (int t = 0; t <= n_zen; ++t)
            range.thetaValues.push_back(DegToRad(theta_deg[t]));
        std::sort(range.thetaValues.begin(), range.thetaValues.end());
        range.isNonUniform = true;
        range.nZenith = n_zen;
        range.zenithStart = range.thetaValues.front();
        range.zenithEnd = range.thetaValues.back();
        range.zenithStep = (range.zenithEnd - range.zenithStart) / n_zen;
    }
    Light light;   // Tracer::SetIncidentLight (Tracer.cpp:124-131)
    light.direction = Point3f(0, 0, -1);
    light.polarizationBasis = Point3f(0, 1, 0);
    range.ComputeSphereDirections(light);
    for (int t = 0; t <= n_zen; ++t)
    {
        theta[t] = range.GetZenith(t);
        if (dcos2pi)
            dcos2pi[t] = range.Compute2PiDcos(t);
    }
    for (int p = 0; p < n_az; ++p)
        for (int t = 0; t <= n_zen; ++t)
        {
            const Point3d &v = range.vf[p][t];
            double *o = vf + ((size_t)p * (n_zen + 1) + t) * 3;
            o[0] = v.x; o[1] = v.y; o[2] = v.z;
        }
    if (az_step)
        *az_step = range.azinuthStep;
    return MBS_PO_OK;
}
