// dropin_cache_check.cpp — GPU check of the drop-in's packed-beam cache.
//
// HandlerPO::HandleOrientationsToLocalGpuOnDevice with a nonzero cacheToken
// keeps a chunk's staged beams on the device and reuses them for the next
// call with the same token and orientation range, on whatever grid that call
// has (the reference's variable-phi theta groups, TracerPOTotal.cpp:6567-6693,
// GpuDiffraction.cu:3464-3500 and 4276-4282).  This program, linked against
// the drop-in translation unit (mbs_fast_b200/host/po_boundary.cpp) and the
// reference's sources, traces a column with the reference tracer and
// PrepareBeams, then compares on two grids:
//   token 0 (no cache)  against  token 77: fill, hit, and a hit after a grid
//   change; a call with another range under the same token refills.
// Run with MBS_GPU_TIMING=1 to see cache=fill/hit in the timing lines.  Exit
// code 0 when every result equals the uncached one bit for bit.
#include "HandlerPOTotal.h"
#include "Hexagonal.h"
#include "TracerPOTotal.h"

#include <cmath>
#include <cstdio>
#include <vector>

namespace
{

double max_abs_diff(const Arr2D &a, const Arr2D &b, int nAz, int nZen)
{
    double d = 0.0;
    for (int p = 0; p < nAz; ++p)
        for (int t = 0; t <= nZen; ++t)
        {
            const double *x = a.RawCell(p, t), *y = b.RawCell(p, t);
            for (int k = 0; k < 16; ++k)
                d = std::fmax(d, std::fabs(x[k] - y[k]));
        }
    return d;
}

}  // namespace

int main()
{
    const ::complex ri(1.3116, 0.0);
    Hexagonal particle(ri, 10.0, 20.0);   // --particle 1 20 10
    TracerPOTotal tracer(&particle, 4, "cache_check");
    tracer.m_scattering->m_wave = 0.532;
    Tracks tracks;
    HandlerPOTotal handler(&particle, &tracer.m_incidentLight, 1, 0.532);
    handler.isCoh = true;
    handler.SetFullOnly(true);
    ScatteringRange gridA(0.0, M_PI, 16, 90), gridB(0.0, M_PI, 24, 60);
    handler.SetScatteringSphere(gridA);
    handler.SetTracks(&tracks);
    handler.SetAbsorptionAccounting(false);
    tracer.SetHandler(&handler);

    // 8 orientations through the reference's own tracer and PrepareBeams
    const int n = 8;
    std::vector<PreparedOrientation> prepared(n);
    Scattering *sc = tracer.m_scattering;
    sc->PrepareForParallelTrace();
    HandlerPO local(&particle, &tracer.m_incidentLight, handler.nTheta, sc->m_wave);
    local.ConfigureForThreadLocalPrepare(handler, sc);
    std::vector<Beam> beams;
    for (int i = 0; i < n; ++i)
    {
        particle.Rotate(0.2 + 0.17 * i, 0.1 + 0.09 * i, 0.0);
        sc->FormShadowBeam(beams);
        if (sc->ScatterLight(0, 0, beams))
            local.PrepareBeams(beams, 1.0 / n, prepared[i]);
        beams.clear();
    }

    bool ok = true;
    for (int g = 0; g < 2; ++g)
    {
        const ScatteringRange &grid = g == 0 ? gridA : gridB;
        handler.SetScatteringSphere(grid);
        const int nAz = grid.nAzimuth, nZen = grid.nZenith;
        Arr2D ref(nAz + 1, nZen + 1, 4, 4), refNs(nAz + 1, nZen + 1, 4, 4);
        ref.ClearArr();
        refNs.ClearArr();
        ok = handler.HandleOrientationsToLocalGpuOnDevice(prepared, 0, n, 0, ref, refNs, 1.0, 0.0, 0)
             && ok;
        for (int rep = 0; rep < 2; ++rep)
        {
            Arr2D m(nAz + 1, nZen + 1, 4, 4), mNs(nAz + 1, nZen + 1, 4, 4);
            m.ClearArr();
            mNs.ClearArr();
            ok = handler.HandleOrientationsToLocalGpuOnDevice(prepared, 0, n, 0, m, mNs, 1.0, 0.0, 77)
                 && ok;
            const double d = max_abs_diff(m, ref, nAz, nZen);
            std::printf("grid %d call %d token 77: max |diff| = %.3e\n", g, rep, d);
            ok = ok && d == 0.0;
        }
    }
    // another range under the same token: refilled, equal to the uncached call
    {
        const int nAz = gridB.nAzimuth, nZen = gridB.nZenith;
        Arr2D ref(nAz + 1, nZen + 1, 4, 4), refNs(nAz + 1, nZen + 1, 4, 4);
        Arr2D m(nAz + 1, nZen + 1, 4, 4), mNs(nAz + 1, nZen + 1, 4, 4);
        ref.ClearArr();
        refNs.ClearArr();
        m.ClearArr();
        mNs.ClearArr();
        ok = handler.HandleOrientationsToLocalGpuOnDevice(prepared, 2, 3, 0, ref, refNs, 1.0, 0.0, 0) && ok;
        ok = handler.HandleOrientationsToLocalGpuOnDevice(prepared, 2, 3, 0, m, mNs, 1.0, 0.0, 77) && ok;
        const double d = max_abs_diff(m, ref, nAz, nZen);
        std::printf("range [2,5) token 77: max |diff| = %.3e\n", d);
        ok = ok && d == 0.0;
    }
    std::printf("%s\n", ok ? "OK" : "FAILED");
    return ok ? 0 : 1;
}
