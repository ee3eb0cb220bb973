// unicycle_obstacles.cu — kinematic unicycle among moving circular keep-out
// regions (layout and formulas in model_params.h).  State [x, y, theta, t],
// control [v, omega].  The cost reads the obstacle table as 16-byte vectors.
#include "mppi_core.h"
#include "model_params.h"

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const UnicycleModelParams* p = reinterpret_cast<const UnicycleModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = p->dt;
  float sn, cs;
  sincosf(s[2], &sn, &cs);
  s[0] += control[0] * cs * dt;
  s[1] += control[0] * sn * dt;
  s[2] += control[1] * dt;
  s[3] += dt;
}

__device__ __forceinline__ float unicycle_goal(const float* s, const UnicycleCostParams* c) {
  const float dx = s[0] - c->goal_x, dy = s[1] - c->goal_y;
  return c->w_goal * (dx * dx + dy * dy);
}

__device__ float mppi_stage_cost(const float* s, const float* control,
                                 const uint8_t* model_params_raw, const uint8_t* cost_params_raw) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  const float t = s[3];
  float pen = 0.0f;
  const unsigned n = c->num_obs < MPPI_UNICYCLE_MAX_OBS ? c->num_obs : MPPI_UNICYCLE_MAX_OBS;
  for (unsigned i = 0; i < n; ++i) {
    const float cx = fmaf(c->obs_vx[i], t, c->obs_cx[i]);
    const float cy = fmaf(c->obs_vy[i], t, c->obs_cy[i]);
    const float ex = s[0] - cx, ey = s[1] - cy;
    pen += fmaxf(c->obs_r[i] - sqrtf(ex * ex + ey * ey), 0.0f);
  }
  return unicycle_goal(s, c) + c->w_obs * pen;
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  return c->w_terminal * unicycle_goal(s, c);
}
