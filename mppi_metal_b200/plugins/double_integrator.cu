// double_integrator.cu — CUDA form of the reference's test model
// (shaders/test_user_dynamics.metal:8-43): state [px, py, vx, vy],
// control [ax, ay], dt = 0.1, stage = terminal = px^2 + py^2.
// Compiled by NVRTC into the rollout kernel; the library provides
// "mppi_core.h" (callable ABI) for plugin sources.
#include "mppi_core.h"

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params, uint2 rng_counter,
                              uint32_t rng_seed) {
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = 0.1f;
  s[0] += s[2] * dt;
  s[1] += s[3] * dt;
  s[2] += control[0] * dt;
  s[3] += control[1] * dt;
}

__device__ float mppi_stage_cost(const float* state, const float* control,
                                 const uint8_t* model_params, const uint8_t* cost_params) {
  return state[0] * state[0] + state[1] * state[1];
}

__device__ float mppi_terminal_cost(const float* state, const uint8_t* model_params,
                                    const uint8_t* cost_params) {
  return state[0] * state[0] + state[1] * state[1];
}
