// mppi_launch.h — kernel argument records shared by the host backend
// (csrc/backend.cpp) and the NVRTC-compiled kernels (mppi_kernels.cuh).
// Plain C layout: only pointers, 32/64-bit integers and floats, so the
// struct is identical under g++, nvcc and NVRTC.
#pragma once

#if !defined(__CUDACC_RTC__)
#include <cstdint>
#endif

// Floats in front of the weighted-noise sums of one partial record:
// [block min cost (hi), sum e, sum e^2, sum cost, block min cost (lo), 0, 0, 0].
// Minimum costs travel as pairs hi + lo of floats (the rollout accumulates
// each sample's cost that way), so the rescaling exp(-(m_b - M) / lambda)
// sees their difference unrounded.
#define MPPI_PARTIAL_HEAD 8

// Floats per agent of the combine statistics:
// [min cost (hi), sum e, sum e^2, sum cost, min cost (lo), 0, 0, 0].
#define MPPI_STATS_STRIDE 8

// The learned proposal's network evaluated per agent on the CUDA cores (the
// per-agent form of its forward pass, used where few agents make the
// tensor-core batch kernel latency-bound): layer l's BF16 weights in the
// tensor-core kernels' K-major core-matrix image (rows = outputs), its FP32
// biases, and where the outputs go.  w[0] null = not used.
struct MppiNetRows {
  const uint16_t* w[4];
  const float* b[4];
  uint32_t in;          // padded input width of layer 0 (32)
  uint32_t hidden;      // hidden width (256)
  uint32_t out;         // padded outputs of layer 3 (multiple of 16)
  uint32_t out_stride;  // floats between agents' output rows
  float* out_buf;       // [N][out_stride]: predicted u* then raw log-scales
};

// One launch of the combine (+ optional propagate & shift) kernel.
// Grid = num_agents, one CTA per agent.
struct MppiCombineArgs {
  uint32_t num_agents;
  uint32_t K;
  uint32_t H;
  uint32_t nblk;
  uint32_t pstride;
  uint32_t step_local;  // history row written by the propagate stage
  float lambda;
  uint32_t propagate;   // 1: propagate x with u*[0], write history, shift u_nom
  const uint32_t* step_base;
  const float* partials;
  const float* u_min;
  const float* u_max;
  const uint8_t* model_params;
  uint64_t model_stride;
  float* u_nom;        // [N][H*m] read; shifted in place when propagating
  float* u_out;        // [N][H*m]
  float* diag;         // [N][3]: best cost, mean cost, effective sample size
  float* stats;        // [N][MPPI_STATS_STRIDE] (may be null)
  float* x;            // [N][n] state, propagated in place
  float* hist_states;  // [T][N][n] (may be null)
  float* hist_controls;  // [T][N][m] (may be null)
  float* hist_costs;   // [T][N] (may be null)
  float* terminal;     // [N][n] (may be null)
  // Uneven batches (null for a uniform batch): per-agent sample count,
  // horizon and first partial record; `block` = rollout CTA size.
  const uint32_t* agent_K;
  const uint32_t* agent_H;
  const uint32_t* agent_blk0;
  uint32_t block;
  uint32_t pad0;
  float* hist_ustar;   // [T][N][H*m] the updated sequence u* of every step (may be null)
  // Proposal features of the propagated state, for the next step's network
  // (modules compiled with MPPI_FEATURES_FN; null = none).
  const uint8_t* cost_params;
  uint64_t cost_stride;
  float* features;          // [N][feature_stride]
  uint32_t feature_stride;  // <= MPPI_MAX_FEATURES
  uint32_t pad1;
  // The next step's network output from those features, computed here by
  // the combine's threads (net.w[0] null: by the separate network kernel).
  MppiNetRows net;
};

// One launch of the fused rollout kernel: every agent of the batch, every
// sample of every agent.  Grid = (nblk, num_agents), one thread per sample.
struct MppiRolloutArgs {
  uint32_t num_agents;
  uint32_t K;           // samples per agent
  uint32_t H;           // horizon
  uint32_t nblk;        // CTAs per agent = ceil(K / block)
  uint32_t stage_rows;  // rows of the per-CTA noise staging buffer; >= H*m
                        // stages the whole horizon during the rollout,
                        // fewer regenerates it chunk by chunk afterwards
  uint32_t seed;        // agent a draws with key seed + a
  uint32_t step_local;  // absolute step index = *step_base + step_local
  uint32_t pstride;     // floats per partial record (head + H*m, padded)
  float lambda;
  uint32_t sigma_stride;      // floats between agents' sigma rows (0: shared)
  uint32_t sigma_inv_stride;  // same for sigma_inv
  uint32_t pad0;
  const uint32_t* step_base;  // device word
  const float* x;             // [N][n] current states
  const float* u_nom;         // [N][H*m] nominal controls
  const float* sigma;         // std-devs (diagonal) or Cholesky factor (full)
  const float* sigma_inv;     // Sigma^-1 (diagonal or full) for the control cost
  const float* u_min;         // [m]
  const float* u_max;         // [m]
  const uint8_t* model_params;  // agent a at + a * model_stride
  const uint8_t* cost_params;
  uint64_t model_stride;
  uint64_t cost_stride;
  // Per-sample costs as pairs costs + costs_lo, [N][K] each; null on the
  // closed loops (only single-step inspection calls keep them).
  float* costs;
  float* costs_lo;
  float* partials;  // [N][nblk][pstride]
  // Uneven batches (all null for a uniform batch).  Agent a has agent_K[a]
  // samples, horizon agent_H[a] <= H (nominals keep the stride H*m) and its
  // partial records start at record agent_blk0[a].  The launch walks `work`
  // items (agent, CTA-of-agent): taken from an atomic queue (work_counter,
  // zero at launch) by a persistent grid, or one item per CTA when
  // work_counter is null.
  const uint32_t* agent_K;
  const uint32_t* agent_H;
  const uint32_t* agent_blk0;
  const uint2* work;
  uint32_t* work_counter;
  uint32_t num_work;
  uint32_t pad1;
  // Learned proposal (read by modules compiled with MPPI_PROPOSAL; prop_out
  // null = plain MPPI).  Samples k < prop_count of agent a draw
  //   eps_t = (mu_t - u_nom_t) + exp(clamp(s, prop_ls_min, prop_ls_max)) * n_t
  // with mu_t[d] = prop_out[a * prop_stride + t * m + d] (the network's
  // predicted u*) and s[d] = prop_out[a * prop_stride + prop_ls_offset + d];
  // the other samples draw the plain eps_t = sigma * n_t.
  // The network may predict fewer steps than the horizon: entries j >=
  // prop_ls_offset (= its H * m) of the sequence get no mean shift.
  const float* prop_out;
  uint32_t prop_stride;
  uint32_t prop_count;
  uint32_t prop_ls_offset;
  float prop_ls_min;
  float prop_ls_max;
  uint32_t pad2;
  // Combine fused into the rollout (uniform batches; null = the separate
  // combine kernel runs).  Every CTA counts itself done in agent_done[agent]
  // once its partial record is written; the last CTA of an agent runs that
  // agent's combine with `comb` and sets the count back to zero, so the
  // words are zero between launches.  No CTA waits for another.
  uint32_t* agent_done;  // [N]
  MppiCombineArgs comb;
};


// Proposal features of state rows: row r is a state of agent r % agents_mod
// (its parameter blobs), out[r][0..out_stride) = the plugin's feature
// callable (entries it does not set are zero).
struct MppiFeaturesArgs {
  uint32_t rows;
  uint32_t agents_mod;
  uint32_t x_stride;    // floats between state rows
  uint32_t out_stride;  // floats between feature rows, <= MPPI_MAX_FEATURES
  const float* x;
  const uint8_t* model_params;
  const uint8_t* cost_params;
  uint64_t model_stride;
  uint64_t cost_stride;
  float* out;
};

// Proposal features and the per-agent network of state rows (the first step
// of a loop whose combines evaluate the network): one CTA per row.
struct MppiProposalRowsArgs {
  MppiFeaturesArgs f;
  MppiNetRows net;
  uint32_t given_features;  // 1: read the features from f.out instead (timing)
  uint32_t pad0;
};

// Normalised weights from the per-sample costs and the combine statistics
// (inspection path; the control update does not need them materialised).
struct MppiWeightsArgs {
  uint32_t num_agents;
  uint32_t K;
  float lambda;
  uint32_t pad0;
  const float* costs;     // [N][K] hi parts
  const float* costs_lo;  // [N][K] lo parts
  const float* stats;     // [N][MPPI_STATS_STRIDE]
  float* weights;         // [N][K]
};

// Noise of samples [k0, k0 + count) of one agent, every time step.
struct MppiNoiseArgs {
  uint32_t k0;
  uint32_t count;
  uint32_t H;
  uint32_t key;
  uint32_t step;
  uint32_t pad0;
  const float* sigma;  // this agent's sigma row
  float* normals;      // [count][H*m] (may be null)
  float* eps;          // [count][H*m] (may be null)
};
