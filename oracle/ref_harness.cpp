// ref_harness.cpp — TEST INFRASTRUCTURE (the checker), not product code.
//
// Drives MBS-fast's own CPU double diffraction path, compiled from the
// reference sources by oracle/Makefile into oracle/_ref/libmbs_ref.so, so the
// tests and the bench's CPU baseline can run the reference on the same inputs
// as the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load this library.
//
//   mbs_ref_run      phase 1 (trace + PrepareBeams) and phase 2 (CPU
//                    diffraction) of TracerPOTotal::TraceWeightedOrientations
//                    (reference src/scattering/TracerPOTotal.cpp:5815-5898 and
//                    :5954-5995), timed separately.
//   mbs_ref_batch    phase 2 only, on an mbs_po_beams batch rebuilt into
//                    PreparedOrientation records, so the reference evaluates
//                    exactly the beams the CUDA path sees.
//   mbs_ref_fixed    the fixed-orientation path HandlerPO::HandleBeams
//                    (HandlerPO.cpp:1102-1608) for one orientation.
//   mbs_ref_jones_kat  the reference's Jones->Mueller known-answer check
//                    (tests/test_mueller_direct.cpp), returning both results.
//   mbs_ref_orientations  the Owen-scrambled Sobol orientations of
//                    TracerPOTotal::TraceFromSobolSeed over the particle's
//                    symmetry domain, from the reference's own Sobol2D and
//                    particle classes (so the reference arm of the bench needs
//                    nothing from this repository's producer).
#include "mbs_po_b200.h"

#include "HandlerPOTotal.h"
#include "Hexagonal.h"
#include "Bullet.h"
#include "Droxtal.h"
#include "ConcaveHexagonal.h"
#include "HexagonalAggregate.h"
#include "TracerPOTotal.h"
#include "Mueller.hpp"
#include "Sobol.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

extern "C" {

// Same field layout as mbs_host_config in include/mbs_host.h.
typedef struct mbs_ref_config {
    int32_t     particle_type;
    double      p[4];
    const char *particle_file;
    double      resize;
    double      ri_re, ri_im;
    int32_t     absorption;
    double      wavelength;
    int32_t     max_reflections;
    int32_t     cutoff_profile;   /* 0 legacy-default, 1 off, 2 safe, 3 balanced, 4 fast */
    int32_t     shadow_off;
    int32_t     legacy_sign;
    int32_t     n_threads;
    int32_t     reference_prepare;        /* unused here */
    double      trace_cutoff_importance;  /* > 0: --trace-cutoff-importance */
    double      beam_cutoff_importance;   /* > 0: --beam-cutoff-importance */
} mbs_ref_config;

typedef struct mbs_ref_gridspec {
    double        zen_start_deg, zen_end_deg;
    int32_t       n_az, n_zen;
    const double *theta_deg;   /* optional non-uniform zenith grid [n_zen+1] */
} mbs_ref_gridspec;

}  // extern "C"

namespace
{

struct RefSetup
{
    std::unique_ptr<Particle> particle;
    std::unique_ptr<TracerPOTotal> tracer;
    std::unique_ptr<HandlerPOTotal> handler;
    Tracks tracks;

    RefSetup(const mbs_ref_config &cfg, const mbs_ref_gridspec &gs)
    {
        // Particle, tracer, handler exactly as src/main.cpp:1674-1775 and
        // :2228-2252 build them for --method po.
        const bool isAbs = cfg.absorption != 0 || cfg.ri_im != 0.0;
        const ::complex ri(cfg.ri_re, isAbs ? cfg.ri_im : 0.0);
        if (cfg.particle_file && cfg.particle_file[0])
        {
            particle.reset(new Particle());
            particle->SetFromFile(cfg.particle_file);
            particle->SetRefractiveIndex(ri);
            if (cfg.resize > 0.0)
                particle->Resize(cfg.resize);
        }
        else if (cfg.particle_type == 1)
            particle.reset(new Hexagonal(ri, cfg.p[1], cfg.p[0]));
        else if (cfg.particle_type == 2)
            particle.reset(new Bullet(ri, cfg.p[1], cfg.p[0],
                                      (cfg.p[1] * std::sqrt(3) * std::tan(DegToRad(62))) / 4));
        else if (cfg.particle_type == 4)
            particle.reset(new Droxtal(ri, DegToRad(32.35), DegToRad(71.81), cfg.p[0]));
        else if (cfg.particle_type == 10)
            particle.reset(new ConcaveHexagonal(ri, cfg.p[1], cfg.p[0], cfg.p[2]));
        else if (cfg.particle_type == 12)
            particle.reset(new HexagonalAggregate(ri, cfg.p[1], cfg.p[0], (int)cfg.p[2]));
        else
            throw std::invalid_argument("unsupported particle type");

        tracer.reset(new TracerPOTotal(particle.get(), cfg.max_reflections, "mbs_ref"));
        tracer->m_scattering->m_wave = cfg.wavelength;
        Scattering *sc = tracer->m_scattering;
        const int profile = cfg.cutoff_profile;
        if (profile == 1)
        {
            sc->restriction = std::numeric_limits<double>::infinity();
            sc->m_traceCutoffJRel = 0.0;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = 0.0;
        }
        else if (profile == 0)
        {
            sc->m_traceCutoffJRel = 1e-7;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = 0.0;
        }
        else
        {
            sc->m_traceCutoffJRel = 0.0;
            sc->m_traceCutoffAreaRel = 0.0;
            sc->m_traceCutoffImportanceRel = profile == 2 ? 1e-12 : (profile == 3 ? 1e-10 : 1e-8);
            sc->restriction = profile == 2 ? 1e8 : (profile == 3 ? 1e5 : 1e3);
        }
        tracer->shadowOff = cfg.shadow_off != 0;
        handler.reset(new HandlerPOTotal(particle.get(), &tracer->m_incidentLight, 1, cfg.wavelength));
        handler->isCoh = true;
        handler->m_legacySign = cfg.legacy_sign != 0;
        if (profile >= 1)
        {
            handler->m_targetEps = 0.0;
            handler->m_beamCutoffJRel = 0.0;
            handler->m_beamCutoffAreaRel = 0.0;
            handler->m_beamCutoffImportanceRel = profile == 1 ? 0.0
                : (profile == 2 ? 1e-10 : (profile == 3 ? 1e-8 : 1e-6));
        }
        ScatteringRange range(DegToRad(gs.zen_start_deg), DegToRad(gs.zen_end_deg), gs.n_az, gs.n_zen);
        if (gs.theta_deg)
        {
            range.thetaValues.clear();
            for (int t = 0; t <= gs.n_zen; ++t)
                range.thetaValues.push_back(DegToRad(gs.theta_deg[t]));
            std::sort(range.thetaValues.begin(), range.thetaValues.end());
            range.isNonUniform = true;
            range.nZenith = gs.n_zen;
            range.zenithStart = range.thetaValues.front();
            range.zenithEnd = range.thetaValues.back();
            range.zenithStep = (range.zenithEnd - range.zenithStart) / gs.n_zen;
        }
        if (cfg.trace_cutoff_importance > 0.0)
            sc->m_traceCutoffImportanceRel = cfg.trace_cutoff_importance;
        if (cfg.beam_cutoff_importance > 0.0)
            handler->m_beamCutoffImportanceRel = cfg.beam_cutoff_importance;
        handler->SetFullOnly(true);
        handler->SetScatteringSphere(range);
        handler->SetTracks(&tracks);
        handler->SetAbsorptionAccounting(isAbs);
        tracer->SetHandler(handler.get());
    }
};

void trace_phase1(RefSetup &s, int n, const double *beta, const double *gamma,
                  const double *alpha, const double *weight, int nThreads,
                  std::vector<PreparedOrientation> &prepared)
{
    prepared.assign(n, PreparedOrientation());
    Scattering *master = s.tracer->m_scattering;
    master->PrepareForParallelTrace();
#pragma omp parallel num_threads(nThreads)
    {
        Particle localParticle = *s.particle;
        Scattering *localScatter = master->CloneFor(&localParticle, &s.tracer->m_incidentLight);
        HandlerPO localHandler(&localParticle, &s.tracer->m_incidentLight,
                               s.handler->nTheta, master->m_wave);
        localHandler.ConfigureForThreadLocalPrepare(*s.handler, localScatter);
        std::vector<Beam> localBeams;
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < n; ++i)
        {
            localParticle.Rotate(beta[i], gamma[i], alpha ? alpha[i] : 0.0);
            if (!s.tracer->shadowOff)
                localScatter->FormShadowBeam(localBeams);
            bool ok = localScatter->ScatterLight(0, 0, localBeams);
            if (ok)
                localHandler.PrepareBeams(localBeams, weight[i], prepared[i]);
            else
                prepared[i].sinZenith = weight[i];
            localBeams.clear();
        }
        delete localScatter;
    }
}

// Phase 2 on the CPU, the OpenMP loop of TracerPOTotal.cpp:5954-5995.
void diffract_phase2(HandlerPO &h, const std::vector<PreparedOrientation> &prepared,
                     int nThreads, Arr2D &M, Arr2D &Mns)
{
    const int nAz = h.m_sphere.nAzimuth;
    const int nZen = h.m_sphere.nZenith;
    const int n = (int)prepared.size();
#pragma omp parallel num_threads(nThreads)
    {
        Arr2D localM(nAz + 1, nZen + 1, 4, 4);
        localM.ClearArr();
        Arr2D localM_ns(nAz + 1, nZen + 1, 4, 4);
        localM_ns.ClearArr();
        std::vector<Arr2DC> localJ, localJ_ns;
        Arr2DC tmp(nAz + 1, nZen + 1, 2, 2);
        tmp.ClearArr();
        localJ.push_back(tmp);
        Arr2DC tmp2(nAz + 1, nZen + 1, 2, 2);
        tmp2.ClearArr();
        localJ_ns.push_back(tmp2);
#pragma omp for schedule(dynamic, 1)
        for (int i = 0; i < n; ++i)
        {
            if (!prepared[i].beams.empty())
                h.HandleBeamsToLocal(prepared[i], localM, localJ, &localJ_ns);
            const double w = prepared[i].sinZenith;
            HandlerPO::AddToMuellerLocal(localJ, w, localM, nAz, nZen);
            HandlerPO::AddToMuellerLocal(localJ_ns, w, localM_ns, nAz, nZen);
            localJ[0].ClearArr();
            localJ_ns[0].ClearArr();
        }
#pragma omp critical(mbs_ref_merge)
        {
            for (int p = 0; p < nAz; ++p)
                for (int t = 0; t <= nZen; ++t)
                {
                    M.insert(p, t, localM(p, t));
                    Mns.insert(p, t, localM_ns(p, t));
                }
        }
    }
}

void export_mueller(const Arr2D &M, int nAz, int nZen, double *out)
{
    if (!out)
        return;
    for (int p = 0; p < nAz; ++p)
        for (int t = 0; t <= nZen; ++t)
        {
            const double *c = M.RawCell(p, t);
            double *o = out + ((size_t)p * (nZen + 1) + t) * 16;
            for (int k = 0; k < 16; ++k)
                o[k] = c[k];
        }
}

int threads_or_all(int n)
{
    return n > 0 ? n : omp_get_max_threads();
}

}  // namespace

extern "C" int mbs_ref_orientations(const mbs_ref_config *cfg, int n, unsigned seed,
                                    double *beta, double *gamma, double *weight)
{
    if (!cfg || n <= 0 || !beta || !gamma || !weight)
        return -1;
    try
    {
        const mbs_ref_gridspec gs = {0.0, 180.0, 1, 1, nullptr};
        RefSetup s(*cfg, gs);
        const Symmetry &sym = s.particle->GetSymmetry();
        // TracerPOTotal.cpp:5476-5488: beta = acos(1 - (1 - cos beta_sym) u),
        // gamma = gamma_sym v, equal weights
        Sobol2D sobol(seed);
        std::vector<double> su, sv;
        sobol.generate(n, su, sv);
        const double cb = std::cos(sym.beta);
        for (int i = 0; i < n; ++i)
        {
            beta[i] = std::acos(1.0 - (1.0 - cb) * su[i]);
            gamma[i] = sym.gamma * sv[i];
            weight[i] = 1.0 / n;
        }
        return 0;
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "mbs_ref_orientations: %s\n", e.what());
        return -1;
    }
}

extern "C" int mbs_ref_run(const mbs_ref_config *cfg, const mbs_ref_gridspec *gs,
                           int n, const double *beta, const double *gamma,
                           const double *alpha, const double *weight,
                           double *M_out, double *Mns_out, double *cext_out,
                           double *trace_seconds, double *diffract_seconds)
{
    try
    {
        RefSetup s(*cfg, *gs);
        const int nThreads = threads_or_all(cfg->n_threads);
        std::vector<PreparedOrientation> prepared;
        auto t0 = std::chrono::steady_clock::now();
        trace_phase1(s, n, beta, gamma, alpha, weight, nThreads, prepared);
        auto t1 = std::chrono::steady_clock::now();
        const int nAz = s.handler->m_sphere.nAzimuth, nZen = s.handler->m_sphere.nZenith;
        Arr2D M(nAz + 1, nZen + 1, 4, 4), Mns(nAz + 1, nZen + 1, 4, 4);
        M.ClearArr();
        Mns.ClearArr();
        diffract_phase2(*s.handler, prepared, nThreads, M, Mns);
        auto t2 = std::chrono::steady_clock::now();
        export_mueller(M, nAz, nZen, M_out);
        export_mueller(Mns, nAz, nZen, Mns_out);
        if (cext_out)
            for (int i = 0; i < n; ++i)
                cext_out[i] = prepared[i].extinctionOt;
        if (trace_seconds)
            *trace_seconds = std::chrono::duration<double>(t1 - t0).count();
        if (diffract_seconds)
            *diffract_seconds = std::chrono::duration<double>(t2 - t1).count();
        return 0;
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "mbs_ref_run: %s\n", e.what());
        return -1;
    }
}

// Rebuild PreparedOrientation records from a flat batch.  Only the fields
// HandleBeamsToLocal reads are set (HandlerPO.cpp:2561-2793).
static void unpack_batch(const mbs_po_beams &b, std::vector<PreparedOrientation> &out)
{
    out.assign(b.n_orient, PreparedOrientation());
    for (int o = 0; o < b.n_orient; ++o)
    {
        PreparedOrientation &po = out[o];
        po.sinZenith = b.orient_weight[o];
        for (int64_t i = b.beam_offsets[o]; i < b.beam_offsets[o + 1]; ++i)
        {
            PreparedBeam pb;
            const int64_t v0 = b.vert_offsets[i];
            const int nv = (int)(b.vert_offsets[i + 1] - v0);
            pb.edgeData.nVertices = nv;
            pb.edgeData.valid = nv >= 3 && nv < BeamEdgeData::MAX_EDGES;
            for (int e = 0; e < nv && e < BeamEdgeData::MAX_EDGES; ++e)
            {
                pb.edgeData.x[e] = b.vx[v0 + e];
                pb.edgeData.y[e] = b.vy[v0 + e];
                pb.edgeData.slope_yx[e] = b.slope_yx[v0 + e];
                pb.edgeData.slope_xy[e] = b.slope_xy[v0 + e];
                pb.edgeData.edge_valid_x[e] = (b.edge_flags[v0 + e] & MBS_PO_EDGE_VALID_X) != 0;
                pb.edgeData.edge_valid_y[e] = (b.edge_flags[v0 + e] & MBS_PO_EDGE_VALID_Y) != 0;
            }
            const double *g = b.beam_geom + (size_t)i * MBS_PO_GEOM_STRIDE;
            pb.bdx = g[0]; pb.bdy = g[1]; pb.bdz = g[2];
            pb.horAx = g[3]; pb.horAy = g[4]; pb.horAz = g[5];
            pb.verAx = g[6]; pb.verAy = g[7]; pb.verAz = g[8];
            pb.cenx = g[9]; pb.ceny = g[10]; pb.cenz = g[11];
            pb.beam_area = g[12];
            pb.pNTx = g[13]; pb.pNTy = g[14]; pb.pNTz = g[15];
            pb.pNPx = g[16]; pb.pNPy = g[17]; pb.pNPz = g[18];
            pb.pnxDTx = g[19]; pb.pnxDTy = g[20]; pb.pnxDTz = g[21];
            pb.pnxDPx = g[22]; pb.pnxDPy = g[23]; pb.pnxDPz = g[24];
            pb.jp00r = g[25]; pb.jp00i = g[26]; pb.jp01r = g[27]; pb.jp01i = g[28];
            pb.jp10r = g[29]; pb.jp10i = g[30]; pb.jp11r = g[31]; pb.jp11i = g[32];
            pb.origBeam.opticalPath = g[33];
            pb.isExternal = (b.beam_flags[i] & MBS_PO_BEAM_EXTERNAL) != 0;
            po.beams.push_back(pb);
        }
    }
}

extern "C" int mbs_ref_batch(const mbs_ref_config *cfg, const mbs_ref_gridspec *gs,
                             const mbs_po_beams *batch, int n_threads,
                             double *M_out, double *Mns_out, double *cext_out,
                             double *seconds)
{
    try
    {
        RefSetup s(*cfg, *gs);
        std::vector<PreparedOrientation> prepared;
        unpack_batch(*batch, prepared);
        const int nAz = s.handler->m_sphere.nAzimuth, nZen = s.handler->m_sphere.nZenith;
        Arr2D M(nAz + 1, nZen + 1, 4, 4), Mns(nAz + 1, nZen + 1, 4, 4);
        M.ClearArr();
        Mns.ClearArr();
        auto t0 = std::chrono::steady_clock::now();
        diffract_phase2(*s.handler, prepared, threads_or_all(n_threads), M, Mns);
        auto t1 = std::chrono::steady_clock::now();
        export_mueller(M, nAz, nZen, M_out);
        export_mueller(Mns, nAz, nZen, Mns_out);
        if (cext_out)
            for (int o = 0; o < batch->n_orient; ++o)
                cext_out[o] = s.handler->ComputeForwardExtinctionOt(prepared[o]);
        if (seconds)
            *seconds = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "mbs_ref_batch: %s\n", e.what());
        return -1;
    }
}

// Fixed orientation through HandlerPO::HandleBeams (the reference's CPU-only
// fixed path, HandlerPO.cpp:1102-1608), Jones converted like AddToMueller
// (HandlerPO.cpp:803-822) for a single orientation of weight 1.
class FixedHandler : public HandlerPOTotal
{
public:
    using HandlerPOTotal::HandlerPOTotal;
    const std::vector<Arr2DC> &Jones() const { return m_diffractedMatrices; }
};

extern "C" int mbs_ref_fixed(const mbs_ref_config *cfg, const mbs_ref_gridspec *gs,
                             double beta, double gamma, double alpha,
                             double *M_out, double *seconds)
{
    try
    {
        RefSetup s(*cfg, *gs);
        FixedHandler fh(s.particle.get(), &s.tracer->m_incidentLight, 1, cfg->wavelength);
        fh.isCoh = true;
        fh.m_legacySign = cfg->legacy_sign != 0;
        fh.SetFullOnly(true);
        fh.SetScatteringSphere(s.handler->m_sphere);
        fh.SetTracks(&s.tracks);
        fh.SetAbsorptionAccounting(cfg->absorption != 0 || cfg->ri_im != 0.0);
        fh.SetScattering(s.tracer->m_scattering);
        fh.CleanJ();
        s.particle->Rotate(beta, gamma, alpha);
        std::vector<Beam> beams;
        if (!s.tracer->shadowOff)
            s.tracer->m_scattering->FormShadowBeam(beams);
        s.tracer->m_scattering->ScatterLight(0, 0, beams);
        auto t0 = std::chrono::steady_clock::now();
        fh.HandleBeams(beams, 1.0);
        auto t1 = std::chrono::steady_clock::now();
        const int nAz = fh.m_sphere.nAzimuth, nZen = fh.m_sphere.nZenith;
        Arr2D M(nAz + 1, nZen + 1, 4, 4);
        M.ClearArr();
        HandlerPO::AddToMuellerLocal(fh.Jones(), 1.0, M, nAz, nZen);
        export_mueller(M, nAz, nZen, M_out);
        if (seconds)
            *seconds = std::chrono::duration<double>(t1 - t0).count();
        return 0;
    }
    catch (const std::exception &e)
    {
        std::fprintf(stderr, "mbs_ref_fixed: %s\n", e.what());
        return -1;
    }
}

// Jones -> Mueller: reference AddMuellerFromJones and the legacy Mueller()
// on the analytic samples of tests/test_mueller_direct.cpp:9-24.
extern "C" int mbs_ref_jones_kat(int n, const double *jones /*[n][8]*/, const double *w,
                                 double *direct /*[n][16]*/, double *legacy /*[n][16]*/)
{
    for (int s = 0; s < n; ++s)
    {
        const double *j = jones + 8 * s;
        const complex j00(j[0], j[1]), j01(j[2], j[3]), j10(j[4], j[5]), j11(j[6], j[7]);
        double d[16] = {};
        AddMuellerFromJones(d, j00, j01, j10, j11, w[s]);
        matrixC jm(2, 2);
        jm[0][0] = j00; jm[0][1] = j01; jm[1][0] = j10; jm[1][1] = j11;
        matrix ref = Mueller(jm);
        ref *= w[s];
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c)
            {
                direct[16 * s + 4 * r + c] = d[4 * r + c];
                legacy[16 * s + 4 * r + c] = ref[r][c];
            }
    }
    return 0;
}
