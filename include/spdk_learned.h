/* Learned a-priori troubled-cell indicator (libspdk_cuda.so). No
 * counterpart in the reference, which detects troubles only a posteriori
 * (src/trouble_detection.cpp).
 *
 * A small MLP: input = per element the nodal density and pressure over
 * their element means minus one ((p+1)^d values each) plus, per active
 * direction, the min and max of the two neighbour elements' mean density
 * and mean pressure over the own mean minus one (4 d values); two hidden
 * layers of width 64 with GELU (erf form); sigmoid output = probability
 * that the element is troubled (any sub-cell flagged by NAD/SED/PAD in any
 * slice of the step). Weights and inputs are BF16, every product and sum
 * accumulates in FP32; training keeps FP32 master weights with Adam.
 *
 * Feature rows are BF16 bit patterns (uint16_t), n_in per element, element
 * order as the solver's fields. Device pointers throughout; calls are
 * asynchronous on `stream` unless stated.
 */
#ifndef SPDK_LEARNED_H
#define SPDK_LEARNED_H

#include <stddef.h>
#include <stdint.h>

#include "spdk.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spdk_mlp spdk_mlp;

/* n_in inputs, `hidden` units in both hidden layers (64 in the indicator),
 * weights drawn from a seeded uniform Glorot range, biases zero */
int spdk_mlp_create(int n_in, int hidden, unsigned long long seed, spdk_mlp** out);
int spdk_mlp_destroy(spdk_mlp* m);
/* parameter vector order: W1 [n_in][hidden], b1, W2 [hidden][hidden], b2, w3 [hidden], b3 */
int spdk_mlp_num_params(spdk_mlp* m, int* count);
int spdk_mlp_get_params(spdk_mlp* m, float* host, int count);   /* FP32 master weights (blocking) */
int spdk_mlp_set_params(spdk_mlp* m, const float* host, int count);  /* resets the Adam moments */
/* probabilities p [batch] of feature rows x [batch][n_in] */
int spdk_mlp_forward(spdk_mlp* m, const uint16_t* x, int batch, float* p, void* stream);
/* weighted binary cross-entropy L = sum_s w_s BCE(p_s, y_s) / sum_s w_s and
 * its gradient with respect to the (BF16-rounded) parameters; loss [1],
 * grad [num_params]; deterministic (fixed-order block reduction) */
int spdk_mlp_loss_grad(spdk_mlp* m, const uint16_t* x, const float* y, const float* w, int batch, float* loss,
                       float* grad, void* stream);
/* one Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the batch; loss [1] may be NULL */
int spdk_mlp_train_step(spdk_mlp* m, const uint16_t* x, const float* y, const float* w, int batch, float lr,
                        float* loss, void* stream);

/* feature rows of the solver's current state: x [n_elements][n_in],
 * n_in = 2 (p+1)^d + 4 d (2D p=3: 40) */
int spdk_hydro_feature_size(spdk_hydro* h, int* n_in);
int spdk_hydro_features(spdk_hydro* h, uint16_t* x, size_t count);
/* From the next step on, every step evaluates the indicator on the state
 * at the start of the step and sends the elements with p > threshold
 * straight to the fallback: their sub-cells count as troubled in every
 * slice; NAD/SED/PAD still run on every cell. m = NULL switches it off. The
 * solver keeps the pointer: destroy the MLP after the solver or after
 * switching it off. */
int spdk_hydro_set_indicator(spdk_hydro* h, spdk_mlp* m, float threshold);

#ifdef __cplusplus
}
#endif
#endif /* SPDK_LEARNED_H */
