/*
 * po_oracle.h — TEST INFRASTRUCTURE (the checker), not product code.
 *
 * A plain-C, double-precision restatement of MBS-fast's CPU physical-optics
 * diffraction path over the flat mbs_po_beams batch.  It exists so the tests
 * can check the CUDA library against an independent implementation; the
 * restatement itself is pinned against the reference compiled from its own
 * sources (oracle/_ref/libmbs_ref.so, see ref_harness.cpp).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline use it.
 */
#ifndef PO_ORACLE_H
#define PO_ORACLE_H

#include "mbs_po_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* HandlerPO::HandleBeamsToLocal + AddToMuellerLocal for every orientation of
 * the batch, coherent mode (reference src/handler/HandlerPO.cpp:2561-2796 and
 * :2888-2907).  Adds into M[n_az*(n_zen+1)*16] and, if non-NULL, Mns (sum over
 * non-external beams).  n_threads <= 0 uses all OpenMP threads. */
int po_oracle_diffract(const mbs_po_beams *b, const mbs_po_grid *g,
                       const mbs_po_wave *w, int n_threads,
                       double *M, double *Mns);

/* Coherent Jones sum of one orientation, J[n_az*(n_zen+1)*8] (overwritten):
 * the localJ accumulator of HandleBeamsToLocal before AddToMuellerLocal. */
int po_oracle_jones(const mbs_po_beams *b, const mbs_po_grid *g,
                    const mbs_po_wave *w, int orient, double *J, double *Jns);

/* AddMuellerFromJones (reference src/math/Mueller.hpp:37-87). */
void po_oracle_jones_to_mueller(const double *j /*[8]*/, double weight,
                                double *out /*[16], +=*/);

/* HandlerPO::ComputeForwardExtinctionOt (HandlerPO.cpp:1812-2009). */
double po_oracle_extinction(const mbs_po_beams *b, const mbs_po_wave *w,
                            int orient);

/* Orientation-average writer of HandlerPOTotal::WriteMatricesToFile
 * (reference src/handler/HandlerPOTotal.cpp:23-122, PoleMueller.h): per zenith
 * row the azimuth average with the L(2*phi) rotation (pole rows unrotated and
 * projected), rows[(n_zen+1)*16].  Also returns the scattering cross-section
 * sum_t M11(t)*dcos2pi(t) and the asymmetry parameter
 * g = sum_t cos(theta_t) M11(t) dcos2pi(t) / sum_t M11(t) dcos2pi(t), with
 * theta_t the zenith of row t (zenith 0 is the forward direction). */
int po_oracle_phi_average(const double *M, int n_az, int n_zen,
                          const double *theta, const double *dcos2pi,
                          double *rows, double *csca, double *asym);

/* Incoherent azimuth-summed M11 on a zenith list (already clamped off the
 * poles), the quantity of HandlerPO::DiffractThetasGpu (reference
 * src/cuda/GpuDiffraction.cu:1909-1956, 4780-4970); m11[n] overwritten.
 * singular = 0 drops nearly singular edges as that reference path does;
 * 1 takes their stable quotient like the Mueller path. */
int po_oracle_thetas_m11(const mbs_po_beams *b, const mbs_po_wave *w, int n_az,
                         double az_step, const double *theta, int n, int singular,
                         double *m11);

#ifdef __cplusplus
}
#endif
#endif
