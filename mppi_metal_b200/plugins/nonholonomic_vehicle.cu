// nonholonomic_vehicle.cu — CUDA form of the reference's example model
// (examples/nonholonomic_vehicle/nonholonomic_vehicle.metal:20-91):
// state [x, y, theta, v], control [a, omega]; theta wrapped to [-pi, pi),
// |v| <= v_max; quadratic goal cost plus control effort, 10x terminal.
#include "mppi_core.h"
#include "model_params.h"

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const NonholonomicModelParams* p =
      reinterpret_cast<const NonholonomicModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = p->dt;
  const float theta = s[2], v = s[3];
  s[0] += v * cosf(theta) * dt;
  s[1] += v * sinf(theta) * dt;
  s[2] += control[1] * dt;
  s[3] += control[0] * dt;
  const float pi = 3.1415926535f;
  s[2] = fmodf(s[2] + pi, 2.0f * pi);
  if (s[2] < 0.0f) s[2] += 2.0f * pi;
  s[2] -= pi;
  if (s[3] > p->v_max) s[3] = p->v_max;
  if (s[3] < -p->v_max) s[3] = -p->v_max;
}

__device__ float mppi_stage_cost(const float* s, const float* control,
                                 const uint8_t* model_params_raw, const uint8_t* cost_params_raw) {
  const NonholonomicCostParams* c = reinterpret_cast<const NonholonomicCostParams*>(cost_params_raw);
  const float dx = s[0] - c->x_goal, dy = s[1] - c->y_goal;
  float cost = c->pos_weight * (dx * dx + dy * dy);
  cost += c->control_weight * (control[0] * control[0] + control[1] * control[1]);
  return cost;
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const NonholonomicCostParams* c = reinterpret_cast<const NonholonomicCostParams*>(cost_params_raw);
  const float dx = s[0] - c->x_goal, dy = s[1] - c->y_goal;
  return c->pos_weight * (dx * dx + dy * dy) * 10.0f;
}
