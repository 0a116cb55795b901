// beam_pack.h — flatten the reference's PreparedOrientation records into the
// mbs_po_beams arrays of the C ABI (include/mbs_po_b200.h).
//
// This is the host half of the drop-in boundary.  It replaces the reference's
// GpuBeam packing (src/cuda/GpuDiffraction.cu:273-358 pack_prepared_gpu_beam
// and the OpenMP packing loop :4380-4428): instead of a 1.4 KB fixed
// 32-vertex record per beam, vertices go to CSR arrays and beam scalars to a
// 34-double record.  Every double is copied bit for bit; the packing is
// lossless, which the tests check against the reference's CPU path.
#pragma once

#include "mbs_po_b200.h"
#include "HandlerPO.h"

#include <string>
#include <vector>

struct MbsPackedBeams
{
    std::vector<int64_t> beam_offsets;
    std::vector<double>  orient_weight;
    std::vector<int64_t> vert_offsets;
    std::vector<double>  vx, vy, slope_yx, slope_xy;
    std::vector<uint8_t> edge_flags;
    std::vector<double>  beam_geom;
    std::vector<uint8_t> beam_flags;
    std::vector<double>  beam_raw;
    std::vector<int64_t> abs_offsets;
    std::vector<double>  abs_paths;
    std::vector<double>  extinction_ot;   // PreparedOrientation::extinctionOt
    int max_vertices = 0;

    mbs_po_beams view(bool with_raw) const;
};

// Pack prepared[start, start+count).  Returns MBS_PO_OK, or MBS_PO_EBEAM when
// a beam has no valid edge data (the reference GPU path rejects such a batch
// with "bad-edge-data", GpuDiffraction.cu:4298-4303).
int mbs_pack_prepared(const std::vector<PreparedOrientation> &prepared,
                      int start, int count, bool with_raw,
                      MbsPackedBeams &out, std::string *err);

// Appends one orientation's beams to `part`, whose arrays are plain
// concatenations: vert_offsets and abs_offsets (size n_beams, no closing
// entry) index part's own vertex and absorption-path arrays, and
// beam_offsets, orient_weight and extinction_ot are left to the caller.  The
// per-beam values are those of mbs_pack_prepared; same validity rule.
int mbs_pack_append(const PreparedOrientation &po, bool with_raw, MbsPackedBeams &part,
                    std::string *err);
