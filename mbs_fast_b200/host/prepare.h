// prepare.h — per-orientation beam preparation for the host producer.
//
// PrepareHandler::Prepare produces, from the beams of one traced orientation,
// the same PreparedOrientation as the reference's HandlerPO::PrepareBeams
// (HandlerPO.cpp:1625-1810), field for field and bit for bit, at a fraction of
// its cost.  The reference spends most of PrepareBeams in two places that do
// not depend on the beam being prepared:
//   * PrecomputeEdgeData (Handler.cpp:641-693) takes the edge tolerance from
//     Particle::MaximalDimention(), an all-pairs scan over the unrotated
//     particle's facet vertices, once per beam; the value is fixed per
//     particle, so it is computed once per handler here;
//   * an absorbing particle's internal beam recovers its facet track from the
//     big-integer beam id three times (ComputeOpticalLengths, the absorption
//     paths, ApplyAbsorption: Tracks::RecoverTrack, Tracks.cpp:152-181) with
//     arbitrary-precision division; here it is decoded once per beam, in 64-bit
//     arithmetic whenever the id fits in 64 bits (the reference's routine
//     otherwise), and the optical path at the beam centre, which the
//     absorption paths and ApplyAbsorption both evaluate, is taken once.
// Everything else calls the reference's own member functions.
#pragma once

#include "HandlerPO.h"

#include <vector>

class PrepareHandler : public HandlerPO
{
public:
    using HandlerPO::HandlerPO;

    // Same contract as HandlerPO::PrepareBeams.
    void Prepare(std::vector<Beam> &beams, double sinZenith, PreparedOrientation &out);

    // The facet track of `beam` from its id, first facet first (the
    // reference's Tracks::RecoverTrack); throws the same runtime_error when
    // the id does not decode for the particle.
    static void DecodeTrack(const Beam &beam, int nFacets, std::vector<int> &track);

    // Batch-only preparation (the host producer's): only what the flat batch
    // (beam_pack.cpp) and ComputeForwardExtinctionOt read is computed, bit
    // for bit as above.  Left out: BeamInfo::opticalLengths and the length
    // indices (three internal optical paths per internal beam), the output
    // cross section and M00 of the unabsorbed beam, the original beam's
    // polygon (origBeam keeps J, opticalPath and nActs) and the handler's
    // output-energy statistic.
    void SetBatchOnly(bool on) { m_batchOnly = on; }

private:
    double EdgeTolerance();
    BeamInfo BeamInfoWithTrack(Beam &beam, const std::vector<int> &track, bool internal);
    void EdgeData(const BeamInfo &info, const Beam &beam, BeamEdgeData &ed);

    double m_edgeTolerance = -1.0;
    bool m_batchOnly = false;
};
