/*
 * mppi_driver_c.h — C ABI over mppi_metal::MPPIDriver, for FFI callers
 * (ctypes, cffi, JNI, cgo ...).  One function per public MPPIDriver method
 * (include/mppi_metal/mppi_driver.hpp; reference
 * include/mppi_metal/mppi_driver.hpp:24-91), with the same validation, the
 * same messages and the same success convention: each returns 1 for true and
 * 0 for false, and writes the error text into err when err != NULL
 * (the reference's `std::string* error`).
 */
#ifndef MPPI_B200_DRIVER_C_H
#define MPPI_B200_DRIVER_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mppi_driver mppi_driver;

/* DriverConfig + DriverOptions, flattened (reference mppi_types.hpp:15-62). */
typedef struct mppi_driver_config {
  uint32_t state_dim;
  uint32_t control_dim;
  uint32_t horizon;
  uint32_t sample_count;
  float lambda;
  uint32_t covariance_form;    /* ControlNoiseConfig::CovarianceForm */
  const float* sigma;
  const float* sigma_inv;
  uint32_t noise_control_dim;  /* ControlNoiseConfig::control_dim */
  const float* u_min;
  const float* u_max;
  uint32_t bounds_control_dim; /* ControlBounds::control_dim */
  uint32_t numeric_mode;       /* DriverConfig::NumericMode */
  uint32_t control_cost;       /* DriverOptions::control_cost */
  struct mppi_proposal* proposal;  /* DriverOptions::proposal (may be NULL) */
  uint32_t proposal_samples;       /* DriverOptions::proposal_samples */
  const char* proposal_features;   /* DriverOptions::proposal_features (NULL: default) */
} mppi_driver_config;

/* ModelPluginSpec, flattened (reference mppi_types.hpp:79-101). */
typedef struct mppi_driver_plugin {
  const char* source_path;   /* ModelPluginSpec::user_metallib_path */
  const char* dynamics;      /* CallableNames */
  const char* stage_cost;
  const char* terminal_cost;
  uint64_t model_params_size; /* ParamLayout */
  uint64_t model_params_alignment;
  uint64_t cost_params_size;
  uint64_t cost_params_alignment;
  const char* schema_hash;
  uint64_t seed;             /* RngConfig */
} mppi_driver_plugin;

/* MPPIDriver(const DriverConfig&[, const DriverOptions&]); deep-copies the
 * config arrays.  Returns NULL only when out of memory. */
mppi_driver* mppi_driver_create(const mppi_driver_config* config);
void mppi_driver_destroy(mppi_driver* d);

int mppi_driver_initialize(mppi_driver* d, const mppi_driver_plugin* plugin, char* err,
                           size_t err_len);
int mppi_driver_set_problem_params(mppi_driver* d, const void* model_params,
                                   size_t model_bytes, const void* cost_params,
                                   size_t cost_bytes, char* err, size_t err_len);

/* MPPIDriver::step.  x0 / x0_dim = StateView; u_override may be NULL;
 * diag4 = {best_cost, mean_cost, effective_sample_size, converged} or NULL. */
int mppi_driver_step(mppi_driver* d, const float* x0, uint32_t x0_dim, const float* u_override,
                     uint32_t override_horizon, uint32_t override_control_dim,
                     const void* model_override, size_t model_override_bytes,
                     const void* cost_override, size_t cost_override_bytes, float* u_next_out,
                     uint32_t out_horizon, uint32_t out_control_dim, float* diag4, char* err,
                     size_t err_len);

int mppi_driver_reset(mppi_driver* d, char* err, size_t err_len);
int mppi_driver_reset_nominal(mppi_driver* d, const float* u_nominal, uint32_t horizon,
                              uint32_t control_dim, char* err, size_t err_len);

/* MPPIDriver::simulate. */
int mppi_driver_simulate(mppi_driver* d, uint32_t num_steps, const float* x0, uint32_t x0_dim,
                         const float* u_override, uint32_t override_horizon,
                         uint32_t override_control_dim, const void* model_override,
                         size_t model_override_bytes, const void* cost_override,
                         size_t cost_override_bytes, float* states_out, float* controls_out,
                         float* costs_out, uint32_t results_num_steps, char* err,
                         size_t err_len);

/* MPPIDriver::simulate_batch (shared params) and its per-agent overload
 * (BatchAgentParams; any of the per-agent pointers may be NULL). */
int mppi_driver_simulate_batch(mppi_driver* d, uint32_t num_agents, uint32_t num_steps,
                               const float* x0_packed, float* states_out, float* controls_out,
                               float* costs_out, float* terminal_states_out,
                               uint32_t results_num_agents, uint32_t results_num_steps,
                               char* err, size_t err_len);
int mppi_driver_simulate_batch_agents(mppi_driver* d, uint32_t num_agents, uint32_t num_steps,
                                      const float* x0_packed, const void* model_params,
                                      size_t model_params_stride, const void* cost_params,
                                      size_t cost_params_stride, const float* sigma,
                                      const uint32_t* sample_counts, const uint32_t* horizons,
                                      float* states_out, float* controls_out,
                                      float* costs_out, float* terminal_states_out,
                                      uint32_t results_num_agents,
                                      uint32_t results_num_steps, char* err, size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* MPPI_B200_DRIVER_C_H */
