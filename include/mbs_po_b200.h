/*
 * mbs_po_b200.h — C ABI of the B200 (sm_100a) physical-optics diffraction library.
 *
 * This is the drop-in boundary under MBS-fast's HandlerPO GPU entry points.
 * The reference compiles those entry points as HandlerPO member functions in
 * src/cuda/GpuDiffraction.cu; here the member functions (see
 * mbs_fast_b200/host/po_boundary.cpp) flatten PreparedOrientation data into
 * the plain arrays below and call this ABI.  No C++ or torch types cross it:
 * plain pointers, sizes and return codes only.
 *
 * Conventions shared by every entry point
 *   - Return 0 (MBS_PO_OK) on success, a negative MBS_PO_E* code on failure.
 *     The library never calls exit(); the message of the last failure of a
 *     context is returned by mbs_po_last_error().
 *   - Mueller outputs are ACCUMULATED (+=), never overwritten, exactly like
 *     the reference's host `localM` accumulator
 *     (reference src/cuda/GpuDiffraction.cu:4751-4766).
 *   - Direction index g = p*(n_zen+1) + t for azimuth bin p in [0, n_az) and
 *     zenith row t in [0, n_zen]; 16 row-major Mueller elements per direction
 *     (reference GpuDiffraction.cu:4755, src/math/PhysMtr.hpp:34-65).
 *   - One context per host thread (mirrors the reference's thread_local
 *     GpuWorkspace, GpuDiffraction.cu:252).  A context is bound to one device.
 */
#ifndef MBS_PO_B200_H
#define MBS_PO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes -------------------------------------------------------- */
#define MBS_PO_OK              0
#define MBS_PO_EINVAL         -1   /* bad argument (null pointer, bad size)          */
#define MBS_PO_EBEAM          -2   /* beam with invalid edge data (nv outside [3,31]) */
#define MBS_PO_ECUDA          -3   /* CUDA runtime error                              */
#define MBS_PO_ENOMEM         -4   /* device or host allocation failed                */
#define MBS_PO_ESTATE         -5   /* grid or wave constants not set                  */
#define MBS_PO_ETIMEOUT       -6   /* a device-side bounded wait gave up              */
#define MBS_PO_ERANGE         -7   /* size beyond a fixed capacity                    */

/* ---- precision of the diffraction kernel ------------------------------- */
#define MBS_PO_FP64            0   /* plain FP64 path (parity with reference FP64)     */
#define MBS_PO_FP32C           1   /* FP32 trig/MAC, FP64 phase + range reduction,
                                      compensated Jones sums                          */

/* ---- per-beam geometry record: doubles, MBS_PO_GEOM_STRIDE per beam -------
 * Field order follows PreparedBeam (reference src/handler/HandlerPO.h:14-47).  */
#define MBS_PO_G_BD            0   /* bdx, bdy, bdz   beam direction                 */
#define MBS_PO_G_HOR           3   /* horAx..z        aperture horizontal axis       */
#define MBS_PO_G_VER           6   /* verAx..z        aperture vertical axis         */
#define MBS_PO_G_CEN           9   /* cenx..z         beam centre                    */
#define MBS_PO_G_AREA         12   /* beam_area                                      */
#define MBS_PO_G_NT           13   /* pNTx..z                                        */
#define MBS_PO_G_NP           16   /* pNPx..z                                        */
#define MBS_PO_G_NXDT         19   /* pnxDTx..z                                      */
#define MBS_PO_G_NXDP         22   /* pnxDPx..z                                      */
#define MBS_PO_G_JP           25   /* jp00r jp00i jp01r jp01i jp10r jp10i jp11r jp11i */
#define MBS_PO_G_OPATH        33   /* origBeam.opticalPath (extinction phase ref.)   */
#define MBS_PO_GEOM_STRIDE    34

/* ---- optional per-beam record for size rescaling (multi-size batches) ----
 * Mirrors GpuBeam::raw*, phasePath, phaseSign (GpuDiffraction.cu:134-140).     */
#define MBS_PO_R_J             0   /* raw J: 00r 00i 01r 01i 10r 10i 11r 11i         */
#define MBS_PO_R_PATH          8   /* phase path (opticalPath or projLenght)         */
#define MBS_PO_R_SIGN          9   /* phase sign (+1 or -1)                          */
#define MBS_PO_RAW_STRIDE     10

/* edge_flags bits (BeamEdgeData::edge_valid_x / edge_valid_y, Handler.h:384-385) */
#define MBS_PO_EDGE_VALID_X    1u
#define MBS_PO_EDGE_VALID_Y    2u
/* beam_flags bits */
#define MBS_PO_BEAM_EXTERNAL   1u  /* PreparedBeam::isExternal                      */

/* A batch of prepared orientations in flat, caller-owned host arrays.
 * Replaces std::vector<PreparedOrientation> (reference HandlerPO.h:50-55). */
typedef struct mbs_po_beams {
    int32_t        n_orient;
    int64_t        n_beams;
    int64_t        n_verts;
    const int64_t *beam_offsets;   /* [n_orient+1] beams of orientation o      */
    const double  *orient_weight;  /* [n_orient]   PreparedOrientation::sinZenith */
    const int64_t *vert_offsets;   /* [n_beams+1]  vertices of beam b           */
    const double  *vx;             /* [n_verts]    BeamEdgeData::x              */
    const double  *vy;             /* [n_verts]    BeamEdgeData::y              */
    const double  *slope_yx;       /* [n_verts]    BeamEdgeData::slope_yx       */
    const double  *slope_xy;       /* [n_verts]    BeamEdgeData::slope_xy       */
    const uint8_t *edge_flags;     /* [n_verts]    MBS_PO_EDGE_VALID_*          */
    const double  *beam_geom;      /* [n_beams*MBS_PO_GEOM_STRIDE]              */
    const uint8_t *beam_flags;     /* [n_beams]    MBS_PO_BEAM_*                */
    /* optional (may be NULL): only read by mbs_po_diffract_multisize */
    const double  *beam_raw;       /* [n_beams*MBS_PO_RAW_STRIDE]               */
    const int64_t *abs_offsets;    /* [n_beams+1]  PreparedBeam::absorptionPaths */
    const double  *abs_paths;      /* [abs_offsets[n_beams]]                    */
} mbs_po_beams;

/* Scattering grid: ScatteringRange (reference src/handler/Handler.h:15-189). */
typedef struct mbs_po_grid {
    int32_t       n_az;     /* nAzimuth: azimuth bins p in [0, n_az)            */
    int32_t       n_zen;    /* nZenith:  zenith rows t in [0, n_zen]            */
    double        az_step;  /* azinuthStep (2*pi/n_az)                          */
    const double *theta;    /* [n_zen+1] GetZenith(t), radians                  */
    const double *vf;       /* [n_az*(n_zen+1)*3] ScatteringRange::vf[p][t]     */
} mbs_po_grid;

/* Wave constants of Handler (reference src/handler/Handler.cpp:102-126). */
typedef struct mbs_po_wave {
    double  wave_index;          /* m_waveIndex = 2*pi/lambda                     */
    double  wavelength;          /* m_wavelength                                  */
    double  compl_wave_re;       /* m_complWave    = -i*lambda/(2*pi)^2           */
    double  compl_wave_im;
    double  inv_compl_wave_re;   /* m_invComplWave = i/lambda                     */
    double  inv_compl_wave_im;
    double  eps1;                /* m_eps1 (edge-coefficient singular threshold)  */
    double  abs_coeff;           /* m_cAbs (absorption; multi-size re-phasing)    */
    double  ot_far_reference_path; /* m_otFarReferencePath (extinction)           */
    double  ot_ping_distance;    /* m_otPingDistance (extinction)                 */
    int32_t legacy_sign;         /* m_legacySign                                  */
    int32_t ot_phase_average;    /* m_otPhaseAverage (extinction)                 */
} mbs_po_wave;

/* Per-call statistics (device timings, work counters). */
typedef struct mbs_po_stats {
    double  kernel_ms;           /* diffraction kernel(s), CUDA events            */
    double  reduce_ms;           /* deterministic partial reduction               */
    double  h2d_ms;              /* host->device copies (host entry points)       */
    double  d2h_ms;              /* device->host copies (host entry points)       */
    int64_t beam_dir_evals;      /* sum over orientations of beams * directions   */
    int64_t vert_dir_evals;      /* sum over beams of nv * directions             */
    int32_t launches;            /* kernels launched by this call                 */
    int32_t n_chunks;            /* orientation chunks (partial accumulators)     */
} mbs_po_stats;

typedef struct mbs_po_ctx    mbs_po_ctx;
typedef struct mbs_po_staged mbs_po_staged;

/* Context lifetime.  Replaces the reference's thread_local GpuWorkspace
 * (GpuDiffraction.cu:188-252). */
int         mbs_po_create(mbs_po_ctx **ctx, int device);
int         mbs_po_destroy(mbs_po_ctx *ctx);
const char *mbs_po_last_error(const mbs_po_ctx *ctx);
const char *mbs_po_version(void);

/* Grid tables, uploaded once per grid (reference GpuDiffraction.cu:4531-4568). */
int mbs_po_set_grid(mbs_po_ctx *ctx, const mbs_po_grid *grid);
/* Wave constants (reference GpuDiffraction.cu:4618-4695 kernel arguments). */
int mbs_po_set_wave(mbs_po_ctx *ctx, const mbs_po_wave *wave);

/* Host-buffer entry point: copy the batch to the device, run the fused
 * diffraction -> coherent Jones sum -> Mueller accumulation, and ADD the
 * weighted Mueller sums into M_accum (and, when non-NULL, the sum over
 * non-external beams into Mns_accum), both [n_az*(n_zen+1)*16] host arrays.
 * Replaces HandlerPO::HandleOrientationsToLocalGpu
 * (reference src/handler/HandlerPO.h:108-120, GpuDiffraction.cu:4159-4778). */
int mbs_po_diffract(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                    double *M_accum, double *Mns_accum, mbs_po_stats *stats);

/* The same call without the host addition: *M_out (and *Mns_out, when
 * Mns_out is non-NULL, for the sums over non-external beams) receive
 * pointers to this call's weighted Mueller sums in the context's
 * page-locked host buffer, [n_az*(n_zen+1)*16] doubles each, valid until
 * the next call on ctx; NULL when the batch holds no beams.  For callers
 * whose accumulators are not one flat array -- the reference's Arr2D keeps
 * every 4x4 cell in its own allocation (src/math/PhysMtr.cpp:6-17) -- so the
 * result reaches them in one pass instead of a flat addition and a second
 * pass.  Drop-in form of HandleOrientationsToLocalGpu
 * (GpuDiffraction.cu:4159-4778, accumulation at 4751-4766). */
int mbs_po_diffract_pinned(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                           const double **M_out, const double **Mns_out, mbs_po_stats *stats);

/* Device-resident path: stage a batch once (H2D + device layout), then run
 * it any number of times.  M_accum_dev / Mns_accum_dev are DEVICE pointers to
 * [n_az*(n_zen+1)*16] doubles, accumulated (+=) on `stream` (a cudaStream_t,
 * NULL for the legacy default stream). */
int mbs_po_stage(mbs_po_ctx *ctx, const mbs_po_beams *beams, mbs_po_staged **out);
int mbs_po_staged_free(mbs_po_ctx *ctx, mbs_po_staged *staged);
/* Re-fill a staged batch with another host batch, in the device memory it
 * already holds (grown in stream order when the new batch needs more).  For
 * producers that stage batch after batch: a ring of staged batches re-filled
 * this way stops allocating once its slots have grown and never frees,
 * where mbs_po_staged_free + mbs_po_stage release memory (cudaFree waits for
 * all work on the device, the next batch's diffraction included) and take
 * it again.  Every diffraction that reads `staged` must have completed
 * before the call (synchronise its stream, or an event recorded after it).
 * On failure the staged batch holds no orientations until it is re-filled.
 * No counterpart in the reference, which uploads every batch anew
 * (GpuDiffraction.cu:4159-4778). */
int mbs_po_restage(mbs_po_ctx *ctx, const mbs_po_beams *beams, mbs_po_staged *staged);
/* A staged batch of n orientations that shares the device records of
 * `src`: orientation i is src's orientation orient_index[i] with weight
 * weight[i] (host arrays); only the orientation table is new.  Orientations
 * may repeat (an orientation set evaluated several times, or re-weighted,
 * without tracing or staging it again).  `src` must outlive the result and
 * not be re-filled while it is in use.  Consecutive entries that do not
 * continue each other's beam range are joined by a weight-0 orientation over
 * the beams between them: empty for a repeat or a backward jump; a forward
 * jump costs the skipped beams' work.  No counterpart in the reference. */
int mbs_po_stage_repeat(mbs_po_ctx *ctx, const mbs_po_staged *src, int n,
                        const int32_t *orient_index, const double *weight,
                        mbs_po_staged **out);
int mbs_po_diffract_staged(mbs_po_ctx *ctx, const mbs_po_staged *staged,
                           int precision, double *M_accum_dev,
                           double *Mns_accum_dev, void *stream,
                           mbs_po_stats *stats);

/* Multi-size scan: the orientations of `beams` at n_scales particle sizes
 * (size factor scales[i] relative to the traced particle), all in one
 * diffraction launch.  Instance i is the batch with vertex coordinates and
 * beam centres times scales[i], beam areas times scales[i]^2 and the Jones
 * matrices re-phased from the unphased records,
 *     J_phased = sign * absorption(s) * J * exp(i wave_index s path)
 * (beam_raw is required; abs_offsets/abs_paths with the absorption
 * coefficient of the wave constants give absorption(s)).  wave_index <= 0
 * uses the context's wave number.  M_accum: n_scales consecutive Mueller
 * planes of [n_az*(n_zen+1)*16] doubles (host), each accumulated +=.
 * Replaces HandlerPO::HandleOrientationsToLocalGpuMultiK (reference
 * GpuDiffraction.cu:3956-4158, src/handler/HandlerPO.h:132-137) and the scaled
 * single-size call HandleOrientationsToLocalGpu(..., scale, waveIndex)
 * (GpuDiffraction.cu:4323-4324). */
int mbs_po_diffract_multisize(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                              const double *scales, int n_scales, double wave_index,
                              int precision, double *M_accum, double *Mns_accum,
                              mbs_po_stats *stats);
/* Device-resident multi-size batch: mbs_po_diffract_staged on it writes
 * mbs_po_staged_sets() consecutive Mueller planes (one per size). */
int mbs_po_stage_multisize(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                           const double *scales, int n_scales, double wave_index,
                           mbs_po_staged **out);
int mbs_po_staged_sets(const mbs_po_staged *staged);

/* Orientation-averaged M11 on a list of zenith angles (radians), summed over
 * the context grid's n_az azimuth bins and over beams INCOHERENTLY:
 *   m11_out[t] = sum_o w_o sum_beams sum_{p<n_az} 0.5 |d|^2 / (n_az + 1)
 * with d the beam's GPU-convention Jones contribution (rotation without the
 * 0.5 factor), zenith angles clamped 1e-6 away from the poles and the
 * stable edge quotient off (zero for |C_e| <= eps1), in FP64.  m11_out[n]
 * (host) is overwritten.  Replaces HandlerPO::DiffractThetasGpu (reference
 * GpuDiffraction.cu:4780-4970, theta_m11_kernel). */
int mbs_po_diffract_thetas(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                           const double *theta_rad, int n, double *m11_out);

/* FFT-phi azimuth interpolation (replaces the upsampling of
 * HandlerPO::HandleOrientationsToLocalGpuFftPhi, reference
 * GpuDiffraction.cu:3206-3320 fft_upsample_phi_arr2d and :3504-3760): a
 * Mueller grid low_dev [n_low][n_rows][16] on n_low equally spaced azimuth
 * bins (device) is interpolated to n_full >= n_low bins and added into
 * full_dev [n_full][n_rows][16] (device, +=): the real part of the
 * zero-padded DFT upsampling, frequencies -(n_low-1)/2 .. n_low/2 (the
 * Nyquist bin of an even n_low kept at +n_low/2), applied as one linear map
 * in FP64.  n_low <= 4096, n_full <= 65535 (MBS_PO_ERANGE beyond). */
int mbs_po_phi_interpolate(mbs_po_ctx *ctx, const double *low_dev, int n_low, int n_rows,
                           double *full_dev, int n_full, void *stream);

/* mbs_po_diffract on the context's grid (n_az azimuth bins), followed on the
 * device by mbs_po_phi_interpolate to n_full bins: M_accum (and Mns_accum)
 * are [n_full][n_zen+1][16] host arrays, accumulated +=.  The low-resolution
 * direct evaluation plus interpolation of the reference's FFT-phi path; the
 * result is an approximation of the direct evaluation on n_full bins whose
 * error depends on how band-limited the pattern is in azimuth. */
int mbs_po_diffract_fft_phi(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                            int n_full, double *M_accum, double *Mns_accum,
                            mbs_po_stats *stats);

/* Post-step on the device: the azimuth-averaged rows of a Mueller grid held
 * in device memory (M_dev, [n_az*(n_zen+1)*16], e.g. the accumulator of
 * mbs_po_diffract_staged), as HandlerPOTotal::WriteMatricesToFile writes them
 * (reference src/handler/HandlerPOTotal.cpp:49-96): per zenith row the mean
 * over azimuth bins of M(p, t) L(2 az_p), az_p = -2 pi p / n_az, polar rows
 * unrotated and projected (PoleMueller ApplyForward / ApplyBackward).
 * rows_out[(n_zen+1)*16] (host).  Also the scattering cross-section
 * C_sca = sum_t M11(t) dcos2pi(t) (dcos2pi[n_zen+1], host: the grid's
 * Compute2PiDcos weights) and the asymmetry parameter
 * g = sum_t cos(theta_t) M11(t) dcos2pi(t) / C_sca, which the reference does
 * not compute.  Only (n_zen+1)*16 doubles cross PCIe instead of the grid. */
int mbs_po_phi_average(mbs_po_ctx *ctx, const double *M_dev, const double *dcos2pi,
                       double *rows_out, double *csca_out, double *asym_out,
                       void *stream);

/* Azimuth-averaged rows of every orientation alone (the per-orientation
 * results the learned orientation proposal trains on; no counterpart in the
 * reference): rows_out[n_orient][(n_zen+1)*16] (host, overwritten), each
 * orientation's Mueller grid times its orientation weight, averaged over
 * azimuth as mbs_po_phi_average does.  The batch runs in groups of
 * orientations whose grids fit about 1 GiB of device memory. */
int mbs_po_orientation_rows(mbs_po_ctx *ctx, const mbs_po_beams *beams, int precision,
                            double *rows_out);

/* Optical-theorem extinction per orientation on the device (weighted by the
 * orientation weight), written to cext_out[n_orient] (host).  Replaces
 * HandlerPO::ComputeForwardExtinctionOt (reference HandlerPO.cpp:1812-2009). */
int mbs_po_extinction(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                      double *cext_out);

/* Upper bound on the orientations per call that fit `mem_fraction` of the
 * device's free memory.  Reads only n_orient, beam_offsets and vert_offsets
 * of `beams` (the other arrays may be NULL).  Replaces
 * HandlerPO::SelectGpuOrientationBatchSize (reference GpuDiffraction.cu:2948-3029). */
int mbs_po_select_batch(mbs_po_ctx *ctx, const mbs_po_beams *beams,
                        int start, int max_count, double mem_fraction,
                        int *count_out);

/* mbs_po_diffract_pinned for a batch staged earlier (mbs_po_stage /
 * mbs_po_restage, one output set): nothing is uploaded.  Serves the
 * drop-in's packed-beam cache (HandleOrientationsToLocalGpuOnDevice with a
 * cacheToken, GpuDiffraction.cu:3464-3500 and 4276-4282), which diffracts
 * the same beams on several grids. */
int mbs_po_diffract_staged_pinned(mbs_po_ctx *ctx, const mbs_po_staged *staged, int precision,
                                  const double **M_out, const double **Mns_out,
                                  mbs_po_stats *stats);

/* Host-side time of the phases of this context's last host-array call
 * (mbs_po_diffract, _pinned, _staged_pinned, _fft_phi, _multisize), ms:
 *   [0] growth of the upload area and staged batch, [1] enqueueing the
 *   host->device copies, [2] record building and its status check,
 *   [3] enqueueing the diffraction, [4] waiting for the device,
 *   [5] handing back the result.  n <= 8 entries.  No counterpart in the
 *   reference (its MBS_GPU_TIMING breakdown, GpuDiffraction.cu:4283-4285). */
int mbs_po_last_profile(const mbs_po_ctx *ctx, double *ms, int n);

/* Helpers of the drop-in's environment knobs: pure functions, the caller
 * passes the environment strings (NULL when unset).
 *   mbs_po_multi_devices  devices one HandleOrientationsToLocalGpu call is
 *       split over: MBS_GPU_MULTI ("0" off, N a limit), MBS_GPU_MULTI_MAX (a
 *       cap), off by default under MPI (gpu_multi_device_count,
 *       GpuDiffraction.cu:595-626).
 *   mbs_po_device_range   device dev's contiguous orientation range of the
 *       split (GpuDiffraction.cu:4224-4226).
 *   mbs_po_eps1_override  the MBS_GPU_EPS1 override of the singular-edge
 *       threshold eps1 (gpu_effective_eps1, GpuDiffraction.cu:498-512).
 *   mbs_po_beam_stats     the MBS_GPU_BEAM_STATS line of a batch
 *       (GpuDiffraction.cu:4354-4443) into buf (MBS_PO_ERANGE if cut). */
int    mbs_po_multi_devices(int work_count, int device_count, const char *multi,
                            const char *multi_max, int under_mpi);
void   mbs_po_device_range(int start, int count, int n_devices, int dev, int *begin, int *sub_count);
double mbs_po_eps1_override(double eps1, const char *value);
int    mbs_po_beam_stats(const mbs_po_beams *beams, char *buf, int len);

/* Allocation-free variant of mbs_po_diffract_staged (no counterpart in the
 * reference).  For callers that cannot allocate device memory when they
 * diffract: callers whose device memory belongs to an external pool or a
 * fixed budget that the library must not draw from, and real-time loops that
 * must not stall on cudaMalloc/cudaFree (both can synchronise the device).  The orientation-chunk partials that
 * mbs_po_diffract_staged keeps in context memory it allocates on demand live
 * here in one fixed device array of MBS_PO_NOALLOC_SCRATCH_BYTES, which
 * every GPU that loads the library holds until the process exits.
 *   - Inputs (the staged batch, grid and wave constants of the context) and
 *     outputs (M_accum_dev / Mns_accum_dev, device arrays of
 *     [n_az*(n_zen+1)*16] doubles, accumulated +=) are the caller's.
 *   - Grids whose partial plane (16 doubles per direction, twice with
 *     Mns_accum_dev) exceeds the array are rejected with MBS_PO_ERANGE; when
 *     the array holds fewer orientation chunks than the default plan uses,
 *     the call runs fewer, larger chunks.
 *   - Throughput: this call uses up to 64 orientation chunks (about 32 work
 *     items per resident CTA; the allocating calls use up to 256, about
 *     128); when fewer chunk planes fit in the array the call runs fewer,
 *     larger chunks and fewer work items.  On the
 *     48 x 1801 grid (11 MB per plane) one chunk fits with no-shadow sums
 *     (240 work items for about 444 resident CTAs: under half the device
 *     busy) and three without.  Grids get the full 64 chunks only up to
 *     4,096 directions (2,048 with no-shadow sums); the largest grid
 *     accepted has 262,142 directions (131,071 with no-shadow sums).
 *   - The first call on a device resolves the array's device address
 *     (cudaGetSymbolAddress) and keeps it for the life of the process; make
 *     that first call before any stream capture.  cudaDeviceReset (or
 *     anything else that destroys the device's primary context) invalidates
 *     the kept address: do not call this entry point after it.
 *   - Every call shares the array and overwrites what the last call left;
 *     calls that overlap on the GPU (other streams, other host threads, other
 *     contexts on the same device) race on it and must be serialised. */
#define MBS_PO_NOALLOC_SCRATCH_BYTES (32u << 20)
int mbs_po_diffract_staged_noalloc(mbs_po_ctx *ctx, const mbs_po_staged *staged,
                                   int precision, double *M_accum_dev,
                                   double *Mns_accum_dev, void *stream);

/* Launch-shape autotuner (project-written; no counterpart in the reference):
 * times each compiled shape of the diffraction kernel (threads per CTA,
 * directions per thread, register budget) on the first max_orient (<= 0:
 * all) orientations of a staged batch, keeps the fastest for `precision` in
 * the context and returns its index in *best; ms_out[v] (may be NULL)
 * receives the kernel time of shape v. */
int mbs_po_autotune(mbs_po_ctx *ctx, const mbs_po_staged *staged, int precision,
                    int max_orient, int *best, double *ms_out, int ms_len);
/* Select a launch shape explicitly (0 = default). */
int mbs_po_set_variant(mbs_po_ctx *ctx, int precision, int variant);

/* Measured FP32 FMA throughput of the context's device in TFLOP/s (independent
 * FFMA chains on every SM), the denominator of the diffraction kernels'
 * roofline fraction.  No counterpart in the reference. */
int mbs_po_probe_fp32_peak(mbs_po_ctx *ctx, double *tflops);
/* Measured FP64 FMA throughput in TFLOP/s (independent DFMA chains), the
 * denominator of the FP64 diffraction kernel's roofline fraction.  No
 * counterpart in the reference. */
int mbs_po_probe_fp64_peak(mbs_po_ctx *ctx, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* MBS_PO_B200_H */
