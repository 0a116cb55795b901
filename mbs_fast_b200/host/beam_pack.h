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

#include <memory>
#include <string>
#include <vector>

// Allocator whose resize() leaves new elements uninitialised: every packed
// array is filled completely by the (parallel) packing pass, so zeroing the
// new elements first would only add a serial pass that also first-touches
// every page on one thread.
template <typename T>
struct MbsNoInitAlloc : std::allocator<T>
{
    template <typename U>
    struct rebind { using other = MbsNoInitAlloc<U>; };
    MbsNoInitAlloc() = default;
    template <typename U>
    MbsNoInitAlloc(const MbsNoInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept { ::new (static_cast<void *>(p)) U; }
    template <typename U, typename... Args>
    void construct(U *p, Args &&...args) { ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...); }
};
template <typename T>
using MbsVec = std::vector<T, MbsNoInitAlloc<T>>;

struct MbsPackedBeams
{
    MbsVec<int64_t> beam_offsets;
    MbsVec<double>  orient_weight;
    MbsVec<int64_t> vert_offsets;
    MbsVec<double>  vx, vy, slope_yx, slope_xy;
    MbsVec<uint8_t> edge_flags;
    MbsVec<double>  beam_geom;
    MbsVec<uint8_t> beam_flags;
    MbsVec<double>  beam_raw;
    MbsVec<int64_t> abs_offsets;
    MbsVec<double>  abs_paths;
    MbsVec<double>  extinction_ot;   // PreparedOrientation::extinctionOt
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
