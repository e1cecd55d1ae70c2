/* pippin_b200: the learned Newton warm start's network (no counterpart in the
 * reference, which warm-starts Newton from the previous step's acceleration,
 * crates/pippin/src/newton.rs:238-245).
 *
 * The network maps 24 contact features to the contact's frame forces
 * (normal, tangent 1, tangent 2): 24 -> 128 -> 128 -> 128 -> 3 with ReLU,
 * stored as one array of 36662 floats (input mean and 1/std, output scale,
 * then W1 [128][24], b1, W2 [128][128], b2, W3, b3, W4 [3][128], b4).
 * Inference runs on the tensor cores in BF16 with FP32 accumulation;
 * training runs FP32 kernels with Adam. All buffers here are host memory. */
#ifndef PIPPIN_B200_MLP_H
#define PIPPIN_B200_MLP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PG_MLP_WEIGHTS 36662 /* floats in a weight array */
#define PG_MLP_PARAMS 36611  /* trained parameters (from W1 on) */

/* Y[n][3] = network(X[n][24]) with the tensor-core inference kernel. */
int pg_mlp_forward(const float* weights, size_t wlen, const float* X, int64_t n, float* Y);

/* Mean squared error over the n samples of the normalised network output
 * against Y / output scale, and its gradient with respect to the 36611
 * trained parameters (same order as the weight array from W1 on), computed
 * by the training kernels. For gradient checks. */
int pg_mlp_loss_grad(const float* weights, size_t wlen, const float* X, const float* Y, int64_t n, float* grad,
                     size_t glen, double* loss);

/* Fits a new network to (X[n][24], Y[n][3]): normalisation from the data,
 * He-uniform initialisation from `seed`, `epochs` passes of Adam over
 * shuffled batches of `batch` samples at learning rate `lr`. Writes the
 * weight array and the mean loss of each epoch (epoch_loss may be NULL). */
int pg_mlp_train(const float* X, const float* Y, int64_t n, int epochs, int batch, float lr, uint64_t seed,
                 float* weights, size_t wlen, double* epoch_loss);

#ifdef __cplusplus
}
#endif

#endif
