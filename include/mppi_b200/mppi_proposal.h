/*
 * mppi_proposal.h — learned sampling proposal for MPPI (C ABI).
 *
 * No reference counterpart: the reference samples every rollout around the
 * warm-started nominal (shaders/mppi_rollout.metal:96-112).  This network
 * predicts, from a per-agent feature vector, the optimised control sequence
 * u* (H x m) and m log-scales s; a proposal-MPPI step then draws a share of
 * its samples around that prediction with standard deviation exp(s), the
 * rest around the warm start as before (mppi_backend_set_proposal).
 *
 * Network: input_dim (<= 32, zero-padded to 32) -> 256 -> 256 -> 256 ->
 * H*m + m, exact-erf GELU after each hidden layer.  BF16 weights and
 * activations, FP32 accumulation on the tcgen05 tensor cores (sm_100a).
 *
 * Training loss (per row, mean over rows and over the H*m entries):
 *   sum_{t,d} [ 0.5 (u*_td - mu_td)^2 exp(-2 c_d) + c_d ] / (H m),
 *   c_d = clamp(s_d, log_scale_min, log_scale_max)
 * -- the Gaussian negative log-likelihood of u* under N(mu, exp(c)^2), so
 * exp(c) learns the network's own prediction error.  Optimiser: Adam
 * (beta 0.9 / 0.999, eps 1e-8) on FP32 master weights.
 *
 * Parameter vector (flat FP32, the order of get/set_params):
 *   W0 [256][32]  b0 [256]   W1 [256][256] b1 [256]
 *   W2 [256][256] b2 [256]   W3 [P][256]   b3 [P]
 * with P = round_up(H*m + m, 16); W0 columns >= input_dim and W3/b3 rows
 * >= H*m + m are padding and stay zero.  Row n of W_l maps the layer's
 * input to its output n (y = W x + b).
 *
 * All x / target / out / index pointers are DEVICE pointers; entry points
 * run on the proposal's own stream and return when their results are ready
 * (train_step without loss_out returns once its kernels are queued).  Every
 * index must be below the row count of x and target.  Return codes are
 * MPPI_OK or an MPPI_ERR_* of mppi_backend.h.
 *
 * Sharing: several backends may run one network at the same time (its
 * weights are only read there), but training it while a backend that has
 * it attached is running races with that backend's reads.
 */
#ifndef MPPI_B200_PROPOSAL_H
#define MPPI_B200_PROPOSAL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mppi_proposal mppi_proposal;

typedef struct mppi_proposal_config {
  uint32_t input_dim;     /* features per row, 1..32 */
  uint32_t horizon;       /* H of the predicted sequence */
  uint32_t control_dim;   /* m; H*m + m <= 256 */
  uint32_t max_batch;     /* rows per training call, >= 1 */
  uint64_t seed;          /* weight initialisation */
  float log_scale_min;    /* clamp of the predicted log-scales */
  float log_scale_max;
} mppi_proposal_config;

mppi_proposal* mppi_proposal_create(const mppi_proposal_config* config, char* err,
                                    size_t err_len);
void mppi_proposal_destroy(mppi_proposal* p);

uint64_t mppi_proposal_param_count(const mppi_proposal* p);
/* Floats between consecutive rows of forward()'s output (P above). */
uint32_t mppi_proposal_output_stride(const mppi_proposal* p);

int mppi_proposal_set_params(mppi_proposal* p, const float* params_host, uint64_t count,
                             char* err, size_t err_len);
int mppi_proposal_get_params(mppi_proposal* p, float* params_host, uint64_t count, char* err,
                             size_t err_len);

/* out[r][0..H*m) = predicted u*, out[r][H*m..H*m+m) = raw log-scales,
 * for r < rows; out has output_stride floats per row. */
int mppi_proposal_forward(mppi_proposal* p, const float* x_dev, uint32_t x_stride,
                          uint32_t rows, float* out_dev, char* err, size_t err_len);

/* Loss and its gradient for rows index[0..rows) of (x, target) (index may be
 * NULL: rows 0..rows).  target rows hold H*m floats.  grads_host receives
 * param_count floats in the parameter order; either output may be NULL. */
int mppi_proposal_gradients(mppi_proposal* p, const float* x_dev, uint32_t x_stride,
                            const float* target_dev, uint32_t target_stride,
                            const uint32_t* index_dev, uint32_t rows, float* loss_out,
                            float* grads_host, char* err, size_t err_len);

/* One Adam step on the same loss (loss_out may be NULL: no host sync). */
int mppi_proposal_train_step(mppi_proposal* p, const float* x_dev, uint32_t x_stride,
                             const float* target_dev, uint32_t target_stride,
                             const uint32_t* index_dev, uint32_t rows, float learning_rate,
                             float* loss_out, char* err, size_t err_len);

/* Milliseconds of the last train_step's kernels (CUDA events). */
float mppi_proposal_last_train_ms(const mppi_proposal* p);

#ifdef __cplusplus
}
#endif

#endif /* MPPI_B200_PROPOSAL_H */
