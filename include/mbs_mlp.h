/*
 * mbs_mlp.h — learned orientation proposal network of the B200 PO library.
 *
 * No counterpart in the reference: MBS-fast averages orientations with plain
 * quasi-random (Sobol) or Euler-grid quadrature.  This network predicts, from
 * the unit quaternion of an orientation, the log of that orientation's
 * contribution to the variance of the orientation-averaged Mueller rows; the
 * importance-sampling proposal built on it (mbs_fast_b200/proposal.py) keeps
 * the average unbiased through its weights.
 *
 * Architecture: 4 -> 128 -> 128 -> 128 -> 1, GELU (erf form) on the hidden
 * layers, BF16 weights and activations on the tensor cores with FP32
 * accumulation, FP32 master parameters and Adam state on the device.
 *
 * Flat FP32 parameter order (MBS_MLP_N_PARAMS floats):
 *   W1[128][4], b1[128], W2[128][128], b2[128], W3[128][128], b3[128],
 *   w4[128], b4[1]      (W[out][in], y = W x + b)
 */
#ifndef MBS_MLP_H
#define MBS_MLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBS_MLP_IN       4
#define MBS_MLP_HIDDEN   128
#define MBS_MLP_N_PARAMS (128 * 4 + 128 + 128 * 128 + 128 + 128 * 128 + 128 + 128 + 1)

typedef struct mbs_mlp mbs_mlp;

/* Network on `device`, parameters initialised from `seed` (uniform
 * +-sqrt(6/fan_in), biases zero). */
int mbs_mlp_create(mbs_mlp **out, int device, uint64_t seed);
int mbs_mlp_destroy(mbs_mlp *net);
const char *mbs_mlp_last_error(const mbs_mlp *net);

/* Watchdog of the tensor-core GEMMs (no counterpart in the reference).
 * Every GEMM waits on its MMA-completion barrier for at most `poll_limit`
 * polls (<= 0: the default 2^22); when the wait runs out the kernel sets the
 * network's device error flag, waits (bounded) for any MMA in flight, frees
 * its tensor memory and returns without storing, and the call fails with
 * "tensor-core barrier wait timed out" (mbs_mlp_last_error); the network
 * stays usable.  skip_mma != 0 is the test hook that exercises this path:
 * the GEMMs then issue no MMA and no commit, so the barrier never completes
 * and no asynchronous operation is pending when the wait gives up. */
int mbs_mlp_set_watchdog(mbs_mlp *net, int poll_limit, int skip_mma);

/* FP32 master parameters, flat order above (host arrays of
 * MBS_MLP_N_PARAMS floats).  set_params also refreshes the BF16 copies and
 * clears the Adam state. */
int mbs_mlp_get_params(mbs_mlp *net, float *params);
int mbs_mlp_set_params(mbs_mlp *net, const float *params);

/* Inference: y[n] = net(q[n][4]) (host arrays). */
int mbs_mlp_forward(mbs_mlp *net, const float *q, int n, float *y);

/* One forward and backward pass of the mean-squared loss
 * L = (1/n) sum_i (net(q_i) - t_i)^2 over the n samples (host arrays);
 * *loss receives L and grad[MBS_MLP_N_PARAMS] dL/dparams (flat order). */
int mbs_mlp_loss_grad(mbs_mlp *net, const float *q, const float *t, int n,
                      float *loss, float *grad);

/* Adam training on the device: `epochs` passes over the n samples in
 * shuffled minibatches of `batch` (seeded), learning rate lr (beta1 0.9,
 * beta2 0.999, eps 1e-8).  *final_loss: mean-squared loss over all samples
 * after training (may be NULL). */
int mbs_mlp_train(mbs_mlp *net, const float *q, const float *t, int n, int epochs,
                  int batch, float lr, uint64_t seed, float *final_loss);

#ifdef __cplusplus
}
#endif
#endif /* MBS_MLP_H */
