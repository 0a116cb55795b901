// beam_pack.cpp — PreparedOrientation -> mbs_po_beams (see beam_pack.h).
#include "beam_pack.h"

#include <cstring>

mbs_po_beams MbsPackedBeams::view(bool with_raw) const
{
    mbs_po_beams v;
    std::memset(&v, 0, sizeof(v));
    v.n_orient = (int32_t)orient_weight.size();
    v.n_beams = (int64_t)beam_flags.size();
    v.n_verts = (int64_t)vx.size();
    v.beam_offsets = beam_offsets.data();
    v.orient_weight = orient_weight.data();
    v.vert_offsets = vert_offsets.data();
    v.vx = vx.data();
    v.vy = vy.data();
    v.slope_yx = slope_yx.data();
    v.slope_xy = slope_xy.data();
    v.edge_flags = edge_flags.data();
    v.beam_geom = beam_geom.data();
    v.beam_flags = beam_flags.data();
    if (with_raw && !beam_raw.empty())
    {
        v.beam_raw = beam_raw.data();
        v.abs_offsets = abs_offsets.data();
        v.abs_paths = abs_paths.data();
    }
    return v;
}

namespace
{

// One beam into slot b of the (already sized) arrays: vertices from v,
// absorption paths from a (advanced past them).  Returns the beam's vertex
// count.
int pack_beam(const PreparedBeam &pb, bool with_raw, MbsPackedBeams &out, int64_t b, int64_t v,
              int64_t &a)
{
    const BeamEdgeData &ed = pb.edgeData;
    const int nv = ed.nVertices;
    out.vert_offsets[b] = v;
    for (int e = 0; e < nv; ++e)
    {
        out.vx[v + e] = ed.x[e];
        out.vy[v + e] = ed.y[e];
        // slope_* is only written by PrecomputeEdgeData where the
        // edge is valid (Handler.cpp:677-690); 0 marks the rest.
        out.slope_yx[v + e] = ed.edge_valid_x[e] ? ed.slope_yx[e] : 0.0;
        out.slope_xy[v + e] = ed.edge_valid_y[e] ? ed.slope_xy[e] : 0.0;
        out.edge_flags[v + e] =
            (uint8_t)((ed.edge_valid_x[e] ? MBS_PO_EDGE_VALID_X : 0u)
                    | (ed.edge_valid_y[e] ? MBS_PO_EDGE_VALID_Y : 0u));
    }
    double *g = &out.beam_geom[(size_t)b * MBS_PO_GEOM_STRIDE];
    g[MBS_PO_G_BD + 0] = pb.bdx;  g[MBS_PO_G_BD + 1] = pb.bdy;  g[MBS_PO_G_BD + 2] = pb.bdz;
    g[MBS_PO_G_HOR + 0] = pb.horAx; g[MBS_PO_G_HOR + 1] = pb.horAy; g[MBS_PO_G_HOR + 2] = pb.horAz;
    g[MBS_PO_G_VER + 0] = pb.verAx; g[MBS_PO_G_VER + 1] = pb.verAy; g[MBS_PO_G_VER + 2] = pb.verAz;
    g[MBS_PO_G_CEN + 0] = pb.cenx; g[MBS_PO_G_CEN + 1] = pb.ceny; g[MBS_PO_G_CEN + 2] = pb.cenz;
    g[MBS_PO_G_AREA] = pb.beam_area;
    g[MBS_PO_G_NT + 0] = pb.pNTx; g[MBS_PO_G_NT + 1] = pb.pNTy; g[MBS_PO_G_NT + 2] = pb.pNTz;
    g[MBS_PO_G_NP + 0] = pb.pNPx; g[MBS_PO_G_NP + 1] = pb.pNPy; g[MBS_PO_G_NP + 2] = pb.pNPz;
    g[MBS_PO_G_NXDT + 0] = pb.pnxDTx; g[MBS_PO_G_NXDT + 1] = pb.pnxDTy; g[MBS_PO_G_NXDT + 2] = pb.pnxDTz;
    g[MBS_PO_G_NXDP + 0] = pb.pnxDPx; g[MBS_PO_G_NXDP + 1] = pb.pnxDPy; g[MBS_PO_G_NXDP + 2] = pb.pnxDPz;
    g[MBS_PO_G_JP + 0] = pb.jp00r; g[MBS_PO_G_JP + 1] = pb.jp00i;
    g[MBS_PO_G_JP + 2] = pb.jp01r; g[MBS_PO_G_JP + 3] = pb.jp01i;
    g[MBS_PO_G_JP + 4] = pb.jp10r; g[MBS_PO_G_JP + 5] = pb.jp10i;
    g[MBS_PO_G_JP + 6] = pb.jp11r; g[MBS_PO_G_JP + 7] = pb.jp11i;
    g[MBS_PO_G_OPATH] = pb.origBeam.opticalPath;
    out.beam_flags[b] = pb.isExternal ? (uint8_t)MBS_PO_BEAM_EXTERNAL : (uint8_t)0;
    if (with_raw)
    {
        // Raw (unabsorbed, unphased) Jones and phase path/sign for
        // size rescaling, as GpuDiffraction.cu:310-330 packs them.
        double *r = &out.beam_raw[(size_t)b * MBS_PO_RAW_STRIDE];
        const Matrix2x2c &J = pb.origBeam.J;
        r[0] = real(J.m11); r[1] = imag(J.m11);
        r[2] = real(J.m12); r[3] = imag(J.m12);
        r[4] = real(J.m21); r[5] = imag(J.m21);
        r[6] = real(J.m22); r[7] = imag(J.m22);
        r[MBS_PO_R_PATH] = pb.isExternal ? pb.origBeam.opticalPath
                                         : pb.info.projLenght;
        double sign = 1.0;
        if (pb.isExternal)
            sign = -sign;
        if (!pb.isExternal && (pb.origBeam.nActs & 1))
            sign = -sign;
        r[MBS_PO_R_SIGN] = sign;
        out.abs_offsets[b] = a;
        for (double path : pb.absorptionPaths)
            out.abs_paths[a++] = path;
    }
    return nv;
}

}  // namespace

int mbs_pack_prepared(const std::vector<PreparedOrientation> &prepared,
                      int start, int count, bool with_raw,
                      MbsPackedBeams &out, std::string *err)
{
    if (start < 0 || count < 0 || start > (int)prepared.size())
    {
        if (err) *err = "bad orientation range";
        return MBS_PO_EINVAL;
    }
    const int nOrient = std::min(count, (int)prepared.size() - start);

    // Pass 1: sizes and validity (GpuDiffraction.cu:4290-4318 does the same
    // scan and rejects beams without valid edge data), and each orientation's
    // first beam, vertex and absorption-path slot.
    std::vector<int64_t> ob(nOrient + 1, 0), ov(nOrient + 1, 0), oa(nOrient + 1, 0);
    for (int oi = 0; oi < nOrient; ++oi)
    {
        int64_t nb = 0, nvt = 0, na = 0;
        for (const PreparedBeam &pb : prepared[start + oi].beams)
        {
            const int nv = pb.edgeData.nVertices;
            if (!pb.edgeData.valid || nv < 3 || nv >= BeamEdgeData::MAX_EDGES)
            {
                if (err) *err = "beam without valid edge data (nv=" + std::to_string(nv) + ")";
                return MBS_PO_EBEAM;
            }
            ++nb;
            nvt += nv;
            na += (int64_t)pb.absorptionPaths.size();
        }
        ob[oi + 1] = ob[oi] + nb;
        ov[oi + 1] = ov[oi] + nvt;
        oa[oi + 1] = oa[oi] + na;
    }
    const int64_t nBeams = ob[nOrient], nVerts = ov[nOrient];

    // every element below is written by pass 2 (uninitialised resize)
    out.beam_offsets.resize(nOrient + 1);
    out.orient_weight.resize(nOrient);
    out.extinction_ot.resize(nOrient);
    out.vert_offsets.resize(nBeams + 1);
    out.vx.resize(nVerts);
    out.vy.resize(nVerts);
    out.slope_yx.resize(nVerts);
    out.slope_xy.resize(nVerts);
    out.edge_flags.resize(nVerts);
    out.beam_geom.resize((size_t)nBeams * MBS_PO_GEOM_STRIDE);
    out.beam_flags.resize(nBeams);
    if (with_raw)
    {
        out.beam_raw.resize((size_t)nBeams * MBS_PO_RAW_STRIDE);
        out.abs_offsets.resize(nBeams + 1);
        out.abs_paths.resize(oa[nOrient]);
    }
    else
    {
        out.beam_raw.clear();
        out.abs_offsets.clear();
        out.abs_paths.clear();
    }

    // Pass 2: the orientations fill disjoint slices, in parallel.
    int maxNv = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(max : maxNv)
    for (int oi = 0; oi < nOrient; ++oi)
    {
        const PreparedOrientation &po = prepared[start + oi];
        int64_t b = ob[oi], v = ov[oi], a = oa[oi];
        out.beam_offsets[oi] = b;
        out.orient_weight[oi] = po.sinZenith;
        out.extinction_ot[oi] = po.extinctionOt;
        for (const PreparedBeam &pb : po.beams)
        {
            const int nv = pack_beam(pb, with_raw, out, b, v, a);
            if (nv > maxNv)
                maxNv = nv;
            v += nv;
            ++b;
        }
    }
    out.max_vertices = maxNv;
    const int64_t b = nBeams, v = nVerts;
    out.beam_offsets[nOrient] = b;
    out.vert_offsets[nBeams] = v;
    if (with_raw)
        out.abs_offsets[nBeams] = (int64_t)out.abs_paths.size();
    return MBS_PO_OK;
}

int mbs_pack_append(const PreparedOrientation &po, bool with_raw, MbsPackedBeams &part,
                    std::string *err)
{
    int64_t nb = 0, nvt = 0, na = 0;
    for (const PreparedBeam &pb : po.beams)
    {
        const int nv = pb.edgeData.nVertices;
        if (!pb.edgeData.valid || nv < 3 || nv >= BeamEdgeData::MAX_EDGES)
        {
            if (err) *err = "beam without valid edge data (nv=" + std::to_string(nv) + ")";
            return MBS_PO_EBEAM;
        }
        ++nb;
        nvt += nv;
        na += (int64_t)pb.absorptionPaths.size();
    }
    int64_t b = (int64_t)part.beam_flags.size(), v = (int64_t)part.vx.size();
    int64_t a = (int64_t)part.abs_paths.size();
    part.vert_offsets.resize(b + nb);
    part.vx.resize(v + nvt);
    part.vy.resize(v + nvt);
    part.slope_yx.resize(v + nvt);
    part.slope_xy.resize(v + nvt);
    part.edge_flags.resize(v + nvt);
    part.beam_geom.resize((size_t)(b + nb) * MBS_PO_GEOM_STRIDE);
    part.beam_flags.resize(b + nb);
    if (with_raw)
    {
        part.beam_raw.resize((size_t)(b + nb) * MBS_PO_RAW_STRIDE);
        part.abs_offsets.resize(b + nb);
        part.abs_paths.resize(a + na);
    }
    for (const PreparedBeam &pb : po.beams)
    {
        const int nv = pack_beam(pb, with_raw, part, b, v, a);
        if (nv > part.max_vertices)
            part.max_vertices = nv;
        v += nv;
        ++b;
    }
    return MBS_PO_OK;
}
