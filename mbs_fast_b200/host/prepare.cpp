// prepare.cpp — PrepareHandler (see prepare.h).  The steps and their order
// follow HandlerPO::PrepareBeams (HandlerPO.cpp:1625-1810),
// HandlerPO::ComputeBeamInfo (:824-878), HandlerPO::ComputeOpticalLengths
// (:1075-1083), Handler::PrecomputeEdgeData (Handler.cpp:641-693),
// Handler::ApplyAbsorption (:220-260) and Tracks::RecoverTrack
// (Tracks.cpp:152-181), so that every field of the result is the same double
// (in batch-only mode, every field the flat batch and the extinction read).
#include "prepare.h"

#include "HandlerPO_fast.h"
#include "Intersection.h"
#include "Mueller.hpp"
#include "Tracks.h"

#include <cfloat>
#include <climits>
#include <cmath>
#include <stdexcept>

void PrepareHandler::DecodeTrack(const Beam &beam, int nFacets, std::vector<int> &track)
{
    track.clear();
    const IdType &id = beam.id;
    if (id.getSign() == BigInteger::negative || id.getLength() > 1)
    {
        Tracks::RecoverTrack(beam, nFacets, track);
        return;
    }
    // The id is sum_i (facet_i + 1) (nFacets + 1)^(i + 1), last facet in the
    // lowest digit; the digit of order 0 is skipped as the reference does
    // (its first step divides the id by the radix).
    const unsigned long long radix = (unsigned long long)nFacets + 1ull;
    unsigned long long rest = (id.getLength() == 0 ? 0ull : (unsigned long long)id.getBlock(0)) / radix;
    const int n = beam.nActs + 1;
    track.resize(n);
    for (int i = 0; i < n; ++i)
    {
        const unsigned long long digit = rest % radix;
        rest = (rest - digit) / radix;
        if (digit < 1 || digit > (unsigned long long)nFacets)
            throw std::runtime_error("beam trajectory id does not decode for the loaded particle "
                                     "(track ids are needed for absorption)");
        track[n - 1 - i] = (int)digit - 1;
    }
}

double PrepareHandler::EdgeTolerance()
{
    // Particle::MaximalDimention scans the unrotated facets, so the value is
    // the same for every orientation of the particle.
    if (m_edgeTolerance < 0.0)
        m_edgeTolerance = geometry_length_tolerance(m_particle->MaximalDimention());
    return m_edgeTolerance;
}

BeamInfo PrepareHandler::BeamInfoWithTrack(Beam &beam, const std::vector<int> &track, bool internal)
{
    BeamInfo info;
    info.normal = beam.Normal();
    info.normald = Point3d(info.normal.cx, info.normal.cy, info.normal.cz);
    info.order = DotProduct(info.normal, beam.direction) > 0;
    info.isBad = false;
    m_isBadBeam = false;
    ComputeCoordinateSystemAxes(info.normald, info.horAxis, info.verAxis);
    info.center = beam.Center();
    info.projectedCenter = ChangeCoordinateSystem(info.horAxis, info.verAxis,
                                                  info.normald, info.center);
    if (internal && !m_batchOnly)
    {
        for (int i = 0; i < 3; ++i)
            info.opticalLengths[i] = m_scattering->ComputeInternalOpticalPath(beam, beam.arr[i], track);
        ComputeLengthIndices(beam, info);
    }
    info.area = beam.Area();
    info.projLenght = beam.opticalPath + DotProductD(info.center, beam.direction);
    info.beamBasis = CrossProduct(beam.polarizationBasis, beam.direction);
    const double basisLength = Length(info.beamBasis);
    if (!(basisLength > EPS_PROJECTION) || !std::isfinite(basisLength))
    {
        info.beamBasis = Point3f(0, 0, 0);
        info.isBad = true;
        m_isBadBeam = true;
        ++m_nBadBeams;
    }
    else
    {
        info.beamBasis = info.beamBasis / basisLength;
    }
    return info;
}

void PrepareHandler::EdgeData(const BeamInfo &info, const Beam &beam, BeamEdgeData &ed)
{
    ed.nVertices = 0;
    ed.valid = false;
    if (beam.nVertices < 3 || beam.nVertices >= BeamEdgeData::MAX_EDGES)
        return;
    const int nv = beam.nVertices;
    ed.nVertices = nv;
    ed.valid = true;
    // aperture coordinates, starting from the last vertex
    for (int i = 0; i < nv; ++i)
    {
        const Point3f v = beam.arr[i == 0 ? nv - 1 : i - 1];
        const Point3d p(v.cx, v.cy, v.cz);
        const Point3d q = p - info.normald * DotProductD(info.normald, p);
        ed.x[i] = DotProductD(q, info.horAxis) - info.projectedCenter.x;
        ed.y[i] = DotProductD(q, info.verAxis) - info.projectedCenter.y;
    }
    const double tol = EdgeTolerance();
    for (int i = 0; i < nv; ++i)
    {
        const int in = (i + 1) % nv;
        const double dx = ed.x[in] - ed.x[i];
        const double dy = ed.y[in] - ed.y[i];
        ed.dx[i] = dx;
        ed.dy[i] = dy;
        ed.edge_valid_x[i] = (fabs(dx) >= tol);
        if (ed.edge_valid_x[i])
        {
            ed.slope_yx[i] = dy / dx;
            ed.intercept_y[i] = ed.y[i] - ed.slope_yx[i] * ed.x[i];
        }
        ed.edge_valid_y[i] = (fabs(dy) >= tol);
        if (ed.edge_valid_y[i])
        {
            ed.slope_xy[i] = dx / dy;
            ed.intercept_x[i] = ed.x[i] - ed.slope_xy[i] * ed.y[i];
        }
    }
}

void PrepareHandler::Prepare(std::vector<Beam> &beams, double sinZenith, PreparedOrientation &out)
{
    out.beams.clear();
    out.beams.reserve(beams.size());
    out.sinZenith = sinZenith;
    out.extinctionOt = 0.0;

    const double jRel = (m_beamCutoffJRel >= 0) ? m_beamCutoffJRel : m_targetEps;
    const double areaRel = (m_beamCutoffAreaRel >= 0) ? m_beamCutoffAreaRel : m_targetEps;
    const double importanceRel = m_beamCutoffImportanceRel;
    const bool useCutoff = (jRel > 0.0) || (areaRel > 0.0) || (importanceRel > 0.0);

    // relative cutoffs: maxima over the particle's beams
    double maxJ = 0, maxArea = 0, maxImportance = 0;
    if (useCutoff)
    {
        for (Beam &beam : beams)
        {
            if (beam.lastFacetId != __INT_MAX__)
            {
                const double jn = beam.J.Norm();
                const double ar = beam.Area();
                const double imp = jn * ar;
                if (jn > maxJ) maxJ = jn;
                if (ar > maxArea) maxArea = ar;
                if (imp > maxImportance) maxImportance = imp;
            }
        }
    }
    const double jThreshold = maxJ * jRel;
    const double areaThreshold = maxArea * areaRel;
    const double importanceThreshold = maxImportance * importanceRel;
    int skipped = 0, skippedJ = 0, skippedArea = 0, skippedImportance = 0, candidates = 0;

    double energy = 0;
    std::vector<int> track;
    for (Beam &beam : beams)
    {
        if (isBackScatteringConusEnabled && beam.direction.cz < backScatteringConus)
            continue;
        beam.polarizationBasis = beam.RotateSpherical(-m_incidentLight->direction,
                                                      m_incidentLight->polarizationBasis);
        const bool internal = m_hasAbsorption && HasInternalOpticalPath(beam);
        if (internal)
            DecodeTrack(beam, m_particle->nFacets, track);
        BeamInfo info = BeamInfoWithTrack(beam, track, internal);
        if (info.isBad)
            continue;

        // the unabsorbed beam: all of it, or (batch-only) the fields the
        // batch reads, its Jones matrix, optical path and act count
        Beam originalBeam;
        if (m_batchOnly)
        {
            originalBeam.J = beam.J;
            originalBeam.opticalPath = beam.opticalPath;
            originalBeam.nActs = beam.nActs;
        }
        else
        {
            originalBeam = beam;
        }
        std::vector<double> absorptionPaths;
        if (internal)
        {
            if (m_absorptionPointCount == 1 || beam.nVertices <= 0)
            {
                absorptionPaths.push_back(m_scattering->ComputeInternalOpticalPath(beam, beam.Center(), track));
            }
            else
            {
                const int count = (m_absorptionPointCount == -1)
                    ? beam.nVertices : std::min(m_absorptionPointCount, beam.nVertices);
                for (int i = 0; i < count; ++i)
                    absorptionPaths.push_back(m_scattering->ComputeInternalOpticalPath(
                        beam, beam.arr[(i * beam.nVertices) / count], track));
            }
            // ApplyAbsorption evaluates the same paths at the same points
            double absorption = 0.0;
            for (double path : absorptionPaths)
                absorption += (path > DBL_EPSILON) ? exp(m_cAbs * path) : 1.0;
            const int nSamples = (int)absorptionPaths.size();
            if (nSamples > 0)
                beam.J *= absorption / nSamples;
        }

        if (beam.lastFacetId != __INT_MAX__)
        {
            ++candidates;
            if (!m_batchOnly)
            {
                matrix mm = Mueller(beam.J);
                energy += BeamCrossSection(beam) * mm[0][0] * sinZenith;
            }
            const double jn = beam.J.Norm();
            const double ar = info.area;
            const double imp = jn * ar;
            if (useCutoff)
            {
                const bool smallJ = (jRel > 0 && jn < jThreshold);
                const bool smallArea = (areaRel > 0 && ar < areaThreshold);
                const bool smallImp = (importanceRel > 0 && imp < importanceThreshold);
                if (smallJ || smallArea || smallImp)
                {
                    skipped++;
                    if (smallJ) skippedJ++;
                    if (smallArea) skippedArea++;
                    if (smallImp) skippedImportance++;
                    continue;
                }
            }
        }

        out.beams.emplace_back();
        PreparedBeam &pb = out.beams.back();
        pb.info = info;
        pb.absorptionPaths = absorptionPaths;
        if (beam.lastFacetId != __INT_MAX__ && !m_batchOnly)
        {
            pb.outputCrossSection = BeamCrossSection(originalBeam);
            matrix unabsorbed = Mueller(originalBeam.J);
            pb.outputMueller00 = unabsorbed[0][0];
        }
        EdgeData(info, beam, pb.edgeData);
        PrecomputePolData(beam, info, pb.polData);
        pb.isExternal = (beam.lastFacetId == __INT_MAX__);
        matrixC J_phased = pb.isExternal
            ? beam.J * fast_exp_im(m_waveIndex * beam.opticalPath)
            : beam.J * fast_exp_im(m_waveIndex * info.projLenght);
        if (pb.isExternal)
            J_phased *= -1.0;
        if (!pb.isExternal && (beam.nActs & 1))
            J_phased *= -1.0;
        pb.horAx = info.horAxis.x; pb.horAy = info.horAxis.y; pb.horAz = info.horAxis.z;
        pb.verAx = info.verAxis.x; pb.verAy = info.verAxis.y; pb.verAz = info.verAxis.z;
        pb.normx = info.normald.x; pb.normy = info.normald.y; pb.normz = info.normald.z;
        const Point3d bd(beam.direction.cx, beam.direction.cy, beam.direction.cz);
        pb.bdx = bd.x; pb.bdy = bd.y; pb.bdz = bd.z;
        pb.cenx = info.center.x; pb.ceny = info.center.y; pb.cenz = info.center.z;
        pb.beam_area = info.area;
        pb.pNTx = pb.polData.NTd.x; pb.pNTy = pb.polData.NTd.y; pb.pNTz = pb.polData.NTd.z;
        pb.pNPx = pb.polData.NPd.x; pb.pNPy = pb.polData.NPd.y; pb.pNPz = pb.polData.NPd.z;
        pb.pnxDTx = pb.polData.nxDT.x; pb.pnxDTy = pb.polData.nxDT.y; pb.pnxDTz = pb.polData.nxDT.z;
        pb.pnxDPx = pb.polData.nxDP.x; pb.pnxDPy = pb.polData.nxDP.y; pb.pnxDPz = pb.polData.nxDP.z;
        const complex j00 = J_phased[0][0], j01 = J_phased[0][1];
        const complex j10 = J_phased[1][0], j11 = J_phased[1][1];
        pb.jp00r = real(j00); pb.jp00i = imag(j00);
        pb.jp01r = real(j01); pb.jp01i = imag(j01);
        pb.jp10r = real(j10); pb.jp10i = imag(j10);
        pb.jp11r = real(j11); pb.jp11i = imag(j11);
        if (m_batchOnly)
        {
            pb.origBeam.J = originalBeam.J;
            pb.origBeam.opticalPath = originalBeam.opticalPath;
            pb.origBeam.nActs = originalBeam.nActs;
        }
        else
        {
            pb.origBeam = originalBeam;
        }
    }

    out.extinctionOt = ComputeForwardExtinctionOt(out);
    m_extinctionCrossSectionOt += out.extinctionOt;
    m_hasExtinctionOt = true;
    m_outputEnergy += energy;
    if (m_beamCutoffStatistics)
    {
        m_beamCutoffStatistics->prepareCalls.fetch_add(1, std::memory_order_relaxed);
        m_beamCutoffStatistics->candidates.fetch_add(candidates, std::memory_order_relaxed);
        m_beamCutoffStatistics->kept.fetch_add(candidates - skipped, std::memory_order_relaxed);
        m_beamCutoffStatistics->rejected.fetch_add(skipped, std::memory_order_relaxed);
        m_beamCutoffStatistics->rejectedJones.fetch_add(skippedJ, std::memory_order_relaxed);
        m_beamCutoffStatistics->rejectedArea.fetch_add(skippedArea, std::memory_order_relaxed);
        m_beamCutoffStatistics->rejectedImportance.fetch_add(skippedImportance, std::memory_order_relaxed);
    }
}
