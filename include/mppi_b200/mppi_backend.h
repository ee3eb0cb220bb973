/*
 * mppi_backend.h — C ABI of the B200 (CUDA, sm_100a) MPPI backend.
 *
 * This is the seam the reference keeps between its driver and its GPU code
 * (MarshallVielmetti/mppi_metal src/metal_backend.hpp:22-108, the
 * Objective-C++ MetalBackend class).  Each entry point below names the
 * MetalBackend method it replaces.  Plain C: opaque handle, plain pointers and
 * sizes, int status (0 = success), and an optional caller buffer for the
 * error text (err may be NULL, as the reference's std::string* error may be).
 *
 * Ownership: nothing passed in is retained; device buffers belong to the
 * backend and are released by mppi_backend_destroy.  A backend is not
 * thread-safe; use one per host thread (each owns its CUDA stream).
 *
 * The C++ driver (include/mppi_metal/mppi_driver.hpp) is the public API and
 * calls this layer; tests and benchmarks may call it directly.
 */
#ifndef MPPI_B200_BACKEND_H
#define MPPI_B200_BACKEND_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MPPI_OK 0
#define MPPI_ERR_INVALID 1     /* bad argument / shape / state */
#define MPPI_ERR_PLUGIN 2      /* plugin source missing, unreadable or failing to compile */
#define MPPI_ERR_CALLABLE 3    /* a named callable is not defined by the plugin */
#define MPPI_ERR_CUDA 4        /* CUDA runtime / driver failure */
#define MPPI_ERR_NO_DEVICE 5   /* no usable CUDA device */
#define MPPI_ERR_NOT_INIT 6    /* backend not initialized */

typedef struct mppi_backend mppi_backend;

/* Largest state (floats).  The reference keeps the state in a 128-byte
 * thread-local buffer and silently truncates larger ones
 * (shaders/mppi_core.h:32); each module here sizes that buffer from
 * state_dim instead -- at least 128 bytes, the reference's value, so its
 * plugins see the same MPPI_MAX_STATE_BYTES -- up to this limit. */
#define MPPI_MAX_STATE_DIM 128

/* DriverConfig as the backend needs it (reference mppi_types.hpp:46-62). */
typedef struct mppi_backend_config {
  uint32_t state_dim;
  uint32_t control_dim;
  uint32_t horizon;
  uint32_t sample_count;
  float lambda;
  uint32_t covariance_form; /* 0: sigma = per-dim std-dev; 1: sigma = full covariance */
  const float* sigma;       /* control_dim or control_dim^2 floats */
  const float* sigma_inv;   /* same shape; read only when control_cost != 0 */
  const float* u_min;       /* control_dim */
  const float* u_max;       /* control_dim */
  uint32_t numeric_mode;    /* DriverConfig::NumericMode: 0 = FP32; 1 (kFp16) and 2
                               (kMixed) draw the noise with approximate
                               transcendentals and round it to FP16 (staged in
                               FP16); dynamics, costs, weights and the update
                               stay FP32 */
  uint32_t control_cost;    /* DriverOptions::control_cost */
} mppi_backend_config;

/* ModelPluginSpec (reference mppi_types.hpp:79-101). */
typedef struct mppi_backend_plugin {
  const char* source_path;   /* CUDA source with the __device__ callables */
  const char* dynamics;      /* required */
  const char* stage_cost;    /* NULL or "": library default (0) */
  const char* terminal_cost; /* NULL or "": library default (0) */
  uint64_t model_params_size; /* ParamLayout sizes: every blob bound or */
  uint64_t cost_params_size;  /* overridden later has exactly this size */
  uint64_t seed;              /* RngConfig::seed; the device key is its low 32 bits */
  /* ParamLayout alignments (0 or 1: unspecified) and schema_hash (NULL or
   * "": none).  A plugin that declares its layout with MPPI_PARAM_LAYOUT
   * (mppi_core.h) compiles only when the sizes are equal, each alignment is
   * unspecified or a multiple of the declared one, and the schema is empty or
   * equal to the declared string; otherwise initialize fails with
   * MPPI_ERR_INVALID naming the field. */
  uint64_t model_params_alignment;
  uint64_t cost_params_alignment;
  const char* schema_hash;
} mppi_backend_plugin;

/* Per-agent inputs of a batch (project extension; NULL = shared). */
typedef struct mppi_batch_agents {
  const void* model_params;
  uint64_t model_params_stride; /* bytes between consecutive agents' blobs */
  const void* cost_params;
  uint64_t cost_params_stride;
  const float* sigma;           /* [N][control_dim] or [N][control_dim^2] */
  /* Uneven batches: per-agent sample count (1..sample_count) and horizon
   * (1..horizon); NULL = the configured value for every agent.  Nominals
   * keep the stride horizon * control_dim.  An uneven batch runs as one
   * persistent launch per pass whose grid size and noise staging are chosen
   * by timing candidates on the first run of each shape (the choice does not
   * change any result bit). */
  const uint32_t* sample_counts;
  const uint32_t* horizons;
} mppi_batch_agents;

/* Constructs an empty backend (MetalBackend::MetalBackend, metal_backend.mm:215). */
int mppi_backend_create(mppi_backend** out);
/* Releases the backend and its device memory (MetalBackend::~MetalBackend). */
void mppi_backend_destroy(mppi_backend* b);

/* Compiles the plugin with the library kernels and allocates device state
 * (MetalBackend::initialize, metal_backend.hpp:35-39 / metal_backend.mm:225-573). */
int mppi_backend_initialize(mppi_backend* b, const mppi_backend_plugin* plugin,
                            const mppi_backend_config* config, char* err, size_t err_len);

/* Uploads the bound parameter blobs (MetalBackend::bind_params,
 * metal_backend.hpp:42-46 / metal_backend.mm:579-600).  Sizes must equal the
 * plugin's ParamLayout sizes (0 with a NULL pointer unbinds). */
int mppi_backend_bind_params(mppi_backend* b, const void* model_params, size_t model_bytes,
                             const void* cost_params, size_t cost_bytes, char* err,
                             size_t err_len);

/* One control step: rollout -> weights -> update (MetalBackend::dispatch_rollout,
 * metal_backend.hpp:57-68 / metal_backend.mm:604-741).  Blob overrides with
 * bytes == 0 use the bound params.  diag3 = {best, mean, ESS}; may be NULL. */
int mppi_backend_dispatch_rollout(mppi_backend* b, uint64_t step_index, const float* x0,
                                  const float* u_nominal, const void* model_params,
                                  size_t model_bytes, const void* cost_params,
                                  size_t cost_bytes, float* u_out, float* diag3, char* err,
                                  size_t err_len);

/* Closed loop, one agent (MetalBackend::dispatch_simulation, metal_backend.hpp:72-83
 * / metal_backend.mm:747-929).  History rows are the local steps 0..T-1. */
int mppi_backend_dispatch_simulation(mppi_backend* b, uint32_t num_steps,
                                     uint64_t start_step_index, const float* x0,
                                     const float* u_nominal, const void* model_params,
                                     size_t model_bytes, const void* cost_params,
                                     size_t cost_bytes, float* states_out,
                                     float* controls_out, float* costs_out, char* err,
                                     size_t err_len);

/* Closed loop, N agents (MetalBackend::dispatch_batch_simulation,
 * metal_backend.hpp:88-100 / metal_backend.mm:935-1124).  u_nominal_packed
 * NULL = zeros.  agents NULL = shared params / sigma.  Outputs may be NULL. */
int mppi_backend_dispatch_batch_simulation(mppi_backend* b, uint32_t num_agents,
                                           uint32_t num_steps, uint64_t start_step_index,
                                           const float* x0_packed,
                                           const float* u_nominal_packed,
                                           const mppi_batch_agents* agents, float* states_out,
                                           float* controls_out, float* costs_out,
                                           float* terminal_states_out, char* err,
                                           size_t err_len);

/* Releases per-shape device buffers and cached graphs (MetalBackend::reset,
 * metal_backend.hpp:103). */
int mppi_backend_reset(mppi_backend* b, char* err, size_t err_len);

/* ---- device-resident batch (split form of dispatch_batch_simulation) ------
 * prepare: upload N agents' states / nominals / per-agent inputs;
 * run:     num_steps closed-loop steps on the resident data (no host copies;
 *          captured once into a CUDA graph per shape and replayed);
 * fetch:   download the histories of the last run.
 * dispatch_batch_simulation == prepare + run + fetch. */
int mppi_backend_batch_prepare(mppi_backend* b, uint32_t num_agents, uint32_t num_steps,
                               const float* x0_packed, const float* u_nominal_packed,
                               const mppi_batch_agents* agents, uint32_t want_states,
                               uint32_t want_controls, uint32_t want_costs,
                               uint32_t want_terminal, char* err, size_t err_len);
int mppi_backend_batch_run(mppi_backend* b, uint64_t start_step_index, char* err,
                           size_t err_len);
/* Device time (ms) of the last batch_run: CUDA events recorded on the
 * backend's stream around the closed-loop graph (waits for it to finish). */
int mppi_backend_last_run_ms(mppi_backend* b, float* ms, char* err, size_t err_len);
int mppi_backend_batch_fetch(mppi_backend* b, float* states_out, float* controls_out,
                             float* costs_out, float* terminal_states_out, float* x_out,
                             float* u_nominal_out, char* err, size_t err_len);

/* ---- inspection (parity tests; no reference counterpart) ------------------ */
/* Per-sample costs and weights are kept by single control steps
 * (mppi_backend_dispatch_rollout) only: the closed loops do not write them
 * (an unread store per sample and step), and after one these calls return
 * MPPI_ERR_INVALID.
 * Per-sample costs of the last control step for agents [a0, a0 + n): [n][K]. */
int mppi_backend_last_costs(mppi_backend* b, uint32_t a0, uint32_t n, float* out, char* err,
                            size_t err_len);
/* The same costs exactly as the rollout accumulated them (each a pair of
 * floats, hi + lo, returned as one double): what the weights were computed
 * from. */
int mppi_backend_last_cost_pairs(mppi_backend* b, uint32_t a0, uint32_t n, double* out,
                                 char* err, size_t err_len);
/* Normalised weights of the last control step for agents [a0, a0 + n): [n][K]. */
int mppi_backend_last_weights(mppi_backend* b, uint32_t a0, uint32_t n, float* out,
                              char* err, size_t err_len);
/* Standard normals and shaped noise of samples [k0, k0 + count) of one agent
 * at one step, with the rollout's own sampling code: [count][H][m] each
 * (either may be NULL).  sigma NULL = the configured sigma. */
int mppi_backend_sample_noise(mppi_backend* b, uint64_t step_index, uint32_t agent,
                              uint32_t k0, uint32_t count, const float* sigma,
                              float* normals_out, float* eps_out, char* err, size_t err_len);
/* Mean device time (ms) of the rollout and combine kernels of the prepared
 * batch shape over `iters` back-to-back launches, timed with CUDA events on
 * the backend's stream. */
int mppi_backend_time_passes(mppi_backend* b, uint32_t iters, float* rollout_ms,
                             float* combine_ms, char* err, size_t err_len);
/* Launch geometry chosen for the prepared batch shape (block = samples per
 * rollout CTA); kernels_per_step =
 * kernel launches of one closed-loop control step (the rollout, which runs
 * the combine in each agent's last CTA for uniform batches, or rollout and
 * combine kernels; plus the network when a proposal is attached). */
int mppi_backend_launch_info(mppi_backend* b, uint32_t* block, uint32_t* nblk,
                             uint32_t* stage_rows, uint32_t* smem_bytes,
                             uint32_t* kernels_per_step);
/* Step form of the last launch shape run (chosen by timing on its first
 * run, or pinned by MPPI_B200_FUSED_COMBINE / _SEPARATE_COMBINE / _WS):
 * bit 0 = combine run by each agent's last rollout CTA, bit 1 =
 * warp-specialised rollout; 0 = plain rollout and separate combine kernel.
 * Bit 2 = cooperative rollout: the plugin splits its stage cost
 * (MPPI_STAGE_COST_SPLIT) and the launch would have at most two plain CTAs
 * per SM, so several lanes share each sample, one part of the cost each;
 * chosen by that rule (MPPI_B200_COOP=0 / 1 pins it), not by timing, as its
 * sums run in their own order.
 * No counterpart in the reference, whose step is a fixed sequence of
 * dispatches (src/metal_backend.mm:678-713). */
int mppi_backend_step_form(mppi_backend* b, uint32_t* form);

/* Autotuner result for the prepared uneven batch: persistent grid size
 * (0 = one CTA per work item), number of work items, noise staging rows and
 * the tuned rollout time (ms).  Returns MPPI_ERR_INVALID for uniform batches
 * or before the first run. */
int mppi_backend_tuning_info(mppi_backend* b, uint32_t* grid, uint32_t* num_work,
                             uint32_t* stage_rows, float* rollout_ms);

/* Philox-2x32-10 words computed on the device (known-answer tests). */
int mppi_device_philox(uint64_t n, const uint32_t* ctr0, const uint32_t* ctr1,
                       const uint32_t* key, uint32_t* out_pairs, char* err, size_t err_len);

/* The library's own sine / cosine evaluated on the device (accuracy tests;
 * no counterpart in the reference, whose Metal build uses the platform's
 * fast-math sin / cos): quarter == 0 gives (sin x, cos x) of mppi_sincosf,
 * quarter != 0 gives (sin(pi/2 x), cos(pi/2 x)) of mppi_sincos_quarter, the
 * Box-Muller angle's form. */
int mppi_device_sincos(uint64_t n, const float* x, int quarter, float* sin_out,
                       float* cos_out, char* err, size_t err_len);

/* The library's own natural logarithm (mppi_log, used by Box-Muller) on the
 * device, for accuracy tests; no counterpart in the reference.  Arguments are
 * normal positive floats. */
int mppi_device_log(uint64_t n, const float* x, float* out, char* err, size_t err_len);

/* ---- allocation-free control step --------------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory once running (a fixed-rate control loop, where cudaMalloc /
 * cudaFree can stall and synchronise the device; an application whose device
 * memory is owned and budgeted by another allocator): one control step for
 * one agent, like mppi_backend_dispatch_rollout, but x0 [state_dim],
 * u_nominal [horizon * control_dim], the two parameter blobs (NULL = zeros),
 * u_out [horizon * control_dim] and diag3 [3] are DEVICE pointers the caller
 * owns, and the step's temporary data lives in one static device array of
 * MPPI_NOALLOC_SCRATCH_BYTES that every GPU loading this library keeps
 * until exit.  The call allocates nothing and rejects (MPPI_ERR_INVALID)
 * problems whose scratch (about 4 * (24 + blocks * (8 + horizon *
 * control_dim)) bytes, blocks = ceil(sample_count / 128)) exceeds the
 * array, and backends with a learned proposal attached (this step is plain
 * MPPI only).
 * It computes the same bits as mppi_backend_dispatch_rollout for the same
 * inputs, and keeps no per-sample costs (mppi_backend_last_costs does not
 * see it).
 * Streams: the step runs on the backend's own stream.  The inputs must be
 * complete in device memory before the call (synchronise the stream that
 * wrote them); the call blocks until the step is done, so the outputs are
 * complete on return.  The caller's current device is restored.
 * The first call on a device looks the array's device address up (make it
 * before any stream capture); the address is kept for the process, so a
 * cudaDeviceReset while the library is in use is not supported.  Calls
 * share the array: calls that overlap on the GPU race. */
#define MPPI_NOALLOC_SCRATCH_BYTES (2u << 20)
int mppi_backend_dispatch_rollout_noalloc(mppi_backend* b, uint64_t step_index, const float* x0,
                                          const float* u_nominal, const void* model_params,
                                          const void* cost_params, float* u_out, float* diag3,
                                          char* err, size_t err_len);

/* ---- learned proposal ---------------------------------------------------
 * No counterpart in the reference (its rollouts all sample around the warm
 * start, shaders/mppi_rollout.metal:96-112).  The network is the object of
 * mppi_proposal.h; the plugin supplies its input through a feature callable
 *   __device__ void f(const float* state, const uint8_t* model_params,
 *                     const uint8_t* cost_params, float* features);
 * that writes up to 32 features (the array arrives zeroed).
 *
 * set_features compiles the callable into the module (NULL / "" removes it;
 * feature_dim = features used, 1..32).  features evaluates it on host state
 * rows [rows][state_dim]: row r belongs to agent r % agents_mod, whose blobs
 * come from the prepared batch (agents_mod == its num_agents) or the bound
 * params (agents_mod == 1); out is [rows][feature_dim].
 *
 * set_proposal attaches a network (NULL detaches; the caller keeps ownership
 * and keeps it alive while attached): every later step -- dispatch_rollout,
 * the closed loops and batches -- first evaluates the features of the
 * current states and the network, then draws samples k <
 * proposal_samples of each agent as (mu - u_nom) + exp(clamp(s)) * n around
 * the predicted sequence mu with the predicted log-scales s, and the other
 * samples as before.  Weights, update and warm start are unchanged.  Needs
 * the network's control_dim == control_dim and input_dim <= feature_dim; a
 * network predicting fewer steps than the horizon shifts only those steps
 * (the rest keep the warm start as their mean).  Takes effect at the next
 * prepare.
 *
 * set_record_ustar (next prepare on) makes the batch closed loop keep the
 * updated sequence u* of every step; batch_fetch_ustar copies it out as
 * [num_steps][num_agents][horizon * control_dim] (the training targets of
 * the network; the matching states are the batch's state history). */
struct mppi_proposal; /* include/mppi_b200/mppi_proposal.h */
int mppi_backend_set_features(mppi_backend* b, const char* callable, uint32_t feature_dim,
                              char* err, size_t err_len);
int mppi_backend_features(mppi_backend* b, const float* states, uint32_t rows,
                          uint32_t agents_mod, float* out, char* err, size_t err_len);
int mppi_backend_set_proposal(mppi_backend* b, struct mppi_proposal* proposal,
                              uint32_t proposal_samples, char* err, size_t err_len);
int mppi_backend_set_record_ustar(mppi_backend* b, uint32_t enable, char* err, size_t err_len);
int mppi_backend_batch_fetch_ustar(mppi_backend* b, float* ustar_out, char* err, size_t err_len);
/* The proposal stage alone on the prepared batch's current states (no
 * counterpart in the reference): features [num_agents][32] and network
 * outputs [num_agents][network output stride] (either may be NULL), and
 * whether the network ran per agent (1: on the CUDA cores, batches of at most
 * 512 agents or MPPI_B200_NET_PER_AGENT=1) or as the tensor-core batch
 * kernel (0).  In closed loops the per-agent form runs inside each agent's
 * combine, for the next step's state. */
int mppi_backend_proposal_stage(mppi_backend* b, float* features_out, float* outputs_out,
                                uint32_t* per_agent, char* err, size_t err_len);
/* Device time (CUDA events) of the proposal stage of one pass on the
 * prepared batch: the feature kernel, and the network's forward pass (the
 * tensor-core batch kernel, or the per-agent network on the features
 * already computed). */
int mppi_backend_time_proposal(mppi_backend* b, uint32_t iters, float* features_ms,
                               float* network_ms, char* err, size_t err_len);

/* Compiles a plugin with the library kernels for sm_100a without loading
 * the result (needs no GPU).  log receives the NVRTC log, including ptxas's
 * register / shared-memory / spill report for every kernel. */
int mppi_compile_check(const mppi_backend_plugin* plugin, const mppi_backend_config* config,
                       char* log, size_t log_len, char* err, size_t err_len);
/* The same for the module a learned proposal uses: proposal != 0 compiles
 * the proposal sampling into the rollout, features (may be NULL) names the
 * plugin's feature callable. */
int mppi_compile_check_proposal(const mppi_backend_plugin* plugin,
                                const mppi_backend_config* config, uint32_t proposal,
                                const char* features, char* log, size_t log_len, char* err,
                                size_t err_len);

/* Library version string. */
const char* mppi_b200_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MPPI_B200_BACKEND_H */
