/*
 * mbs_host.h — C ABI of the beam producer: MBS-fast's own host tracer and
 * beam preparation, compiled from the reference sources, handing over each
 * orientation's outgoing beams as an mbs_po_beams batch.
 *
 * This is the caller side of the drop-in boundary.  It runs what the
 * reference's orientation driver runs before it calls the GPU backend
 * (phase 1 of TracerPOTotal::TraceWeightedOrientations,
 * reference src/scattering/TracerPOTotal.cpp:5815-5898): rotate the particle,
 * FormShadowBeam + ScatterLight, HandlerPO::PrepareBeams.  It also exposes
 * the reference's Sobol orientation generator, grid tables and wave constants
 * so that a caller outside the reference CLI builds exactly the inputs the
 * reference would.
 */
#ifndef MBS_HOST_H
#define MBS_HOST_H

#include "mbs_po_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Particle / run configuration, matching the reference CLI options. */
typedef struct mbs_host_config {
    int32_t     particle_type;   /* --particle type: 1 hexagonal column (L, D),
                                    2 bullet (L, D), 4 droxtal (size),
                                    10 concave hexagonal (L, D, depth),
                                    12 hexagonal aggregate (L, D, n)           */
    double      p[4];            /* --particle parameters after the type       */
    const char *particle_file;   /* --pf file (overrides particle_type if set) */
    double      resize;          /* --rs new Dmax for a file particle (0: off) */
    double      ri_re, ri_im;    /* --refractive-index                         */
    int32_t     absorption;      /* --absorption (also on when ri_im != 0)     */
    double      wavelength;      /* --wavelength-um                            */
    int32_t     max_reflections; /* --max-reflections                          */
    int32_t     cutoff_profile;  /* --cutoff-profile: 0 legacy-default, 1 off,
                                    2 safe, 3 balanced, 4 fast (main.cpp:117-226) */
    int32_t     shadow_off;      /* --shadow_off                               */
    int32_t     legacy_sign;     /* --legacy_sign                              */
    int32_t     n_threads;       /* OpenMP threads for tracing (<=0: all)      */
    int32_t     reference_prepare; /* 1: the reference's HandlerPO::PrepareBeams;
                                    0: the producer's restatement of it (same
                                    result bit for bit, edge tolerance and
                                    facet tracks computed once)               */
    double      trace_cutoff_importance; /* --trace-cutoff-importance (> 0:
                                    overrides the profile's, main.cpp:228-229) */
    double      beam_cutoff_importance;  /* --beam-cutoff-importance (> 0:
                                    overrides the profile's, main.cpp:152-153) */
} mbs_host_config;

typedef struct mbs_host_batch mbs_host_batch;

/* Trace and prepare n_orient orientations (beta, gamma, alpha in radians,
 * weight = PreparedOrientation::sinZenith) and pack them.  Returns 0 or a
 * negative MBS_PO_E* code with a message in err. */
int mbs_host_trace(const mbs_host_config *cfg, int n_orient,
                   const double *beta, const double *gamma,
                   const double *alpha, const double *weight,
                   mbs_host_batch **out, char *err, int errlen);
const mbs_po_beams *mbs_host_batch_view(const mbs_host_batch *batch);
/* PreparedOrientation::extinctionOt of orientation o (host, CPU double). */
double mbs_host_batch_extinction(const mbs_host_batch *batch, int o);
/* Seconds spent tracing + preparing (wall clock). */
double mbs_host_batch_trace_seconds(const mbs_host_batch *batch);
/* Time split of the batch's production: out3[0] = seconds in the tracer
 * (rotation, shadow beam, ScatterLight) and out3[1] = seconds in
 * PrepareBeams, both summed over the worker threads; out3[2] = seconds of
 * packing into the flat batch (per-orientation appends summed over the
 * threads, plus the final gather in orientation order). */
int    mbs_host_batch_phase_seconds(const mbs_host_batch *batch, double *out3);
void   mbs_host_batch_free(mbs_host_batch *batch);

/* Particle symmetry (Particle::GetSymmetry): beta and gamma domains. */
int mbs_host_symmetry(const mbs_host_config *cfg, double *beta_sym,
                      double *gamma_sym, double *dmax);
/* Owen-scrambled 2-D Sobol orientations of TracerPOTotal::TraceFromSobolSeed
 * (reference TracerPOTotal.cpp:5465-5492): beta, gamma, weight = 1/n. */
int mbs_host_sobol_orientations(int n, unsigned seed, double beta_sym,
                                double gamma_sym, double *beta, double *gamma,
                                double *weight);
/* Wave constants of a HandlerPO built from cfg (Handler.cpp:102-126). */
int mbs_host_wave(const mbs_host_config *cfg, mbs_po_wave *wave);
/* Grid tables of ScatteringRange(zen_start, zen_end, n_az, n_zen) after
 * ComputeSphereDirections (Handler.h:127-174).  theta_deg (may be NULL)
 * gives a non-uniform zenith grid (LoadThetaGrid) with n_zen+1 values.
 * theta[n_zen+1], vf[n_az*(n_zen+1)*3], dcos2pi[n_zen+1] = Compute2PiDcos. */
int mbs_host_grid(double zen_start_deg, double zen_end_deg, int n_az,
                  int n_zen, const double *theta_deg, double *theta,
                  double *vf, double *dcos2pi, double *az_step);

#ifdef __cplusplus
}
#endif
#endif /* MBS_HOST_H */
