/* C ABI of the surrogate network used by the adaptive energy sampler.
 *
 * No counterpart in the reference: NEGFtrans evaluates transmission on the
 * uniform grid E_i = E1 + (E2-E1)(i-1)/N_E (main.f90:369-375).  The network
 * is a fully connected map width[0] -> ... -> width[L] with GELU on the
 * hidden layers and a linear output layer.  Products use BF16 operands with
 * FP32 accumulation on the tensor cores; parameters are FP32 master values
 * updated by Adam (beta1 = 0.9, beta2 = 0.999, eps = 1e-8).
 *
 * Packed parameter order: W_0 (width[1] x width[0], row-major), b_0
 * (width[1]), W_1, b_1, ...  Data are row-major (sample, feature).  The loss
 * is the weighted mean square error sum w (y - t)^2 / sum w over a batch.
 * All pointers are host pointers; every call blocks until its work is done.
 */
#ifndef NEGF_MLP_H
#define NEGF_MLP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NEGF_MLP_OK 0
#define NEGF_MLP_ERR_ARG (-1)
#define NEGF_MLP_ERR_CUDA (-2)
#define NEGF_MLP_ERR_NOMEM (-3)

typedef struct negf_mlp negf_mlp;

/* widths[0..n_layers]; max_batch bounds the rows of one forward / gradient
 * pass.  Parameters start at zero: set them with negf_mlp_set_params. */
int negf_mlp_create(int32_t n_layers, const int32_t *widths, int32_t max_batch, int32_t device,
                    negf_mlp **out);
int negf_mlp_destroy(negf_mlp *m);

/* Number of packed parameters (floats). */
int64_t negf_mlp_param_count(const negf_mlp *m);

/* Copies the packed parameters in (and resets the Adam moments) or out. */
int negf_mlp_set_params(negf_mlp *m, const float *params);
int negf_mlp_get_params(negf_mlp *m, float *params);

/* y (batch x width[L]) = network(x (batch x width[0])); any batch size. */
int negf_mlp_forward(negf_mlp *m, const float *x, int32_t batch, float *y);

/* Loss and its gradient w.r.t. the packed parameters for one batch
 * (batch <= max_batch) of inputs x, targets t and weights w. */
int negf_mlp_grad(negf_mlp *m, const float *x, const float *t, const float *w, int32_t batch, double *loss,
                  float *grad);

/* `steps` Adam steps with learning rate lr on minibatches of `batch` rows
 * drawn without replacement (a new permutation per epoch, seeded) from the
 * n rows of (x, t, w), all resident on the device; losses[s] (optional)
 * receives the minibatch loss before step s. */
int negf_mlp_train(negf_mlp *m, const float *x, const float *t, const float *w, int64_t n, int32_t batch,
                   int32_t steps, float lr, uint64_t seed, double *losses);

#ifdef __cplusplus
}
#endif
#endif
