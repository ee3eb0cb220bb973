// bicycle_lane.cu — kinematic bicycle tracking a cubic-spline lane centreline
// (layout and formulas in model_params.h).  State [x, y, theta, v, delta],
// control [accel, steer_rate].
#include "mppi_core.h"
#include "model_params.h"

// The blobs this plugin reads (checked against the driver's ParamLayout).
MPPI_PARAM_LAYOUT_OF(BicycleModelParams, BicycleCostParams, "mppi_b200/bicycle_lane/1")

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const BicycleModelParams* p = reinterpret_cast<const BicycleModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = p->dt;
  const float th = s[2], v = s[3], de = s[4];
  float sn, cs;
  mppi_sincosf(th, &sn, &cs);
  s[0] += v * cs * dt;
  s[1] += v * sn * dt;
  s[2] += v / p->wheelbase * tanf(de) * dt;
  s[3] += control[0] * dt;
  s[4] = fminf(fmaxf(de + control[1] * dt, -p->delta_max), p->delta_max);
}

// Lateral, heading and speed errors against the centreline at x.
__device__ __forceinline__ float bicycle_state_cost(const float* s, const BicycleCostParams* c) {
  const float xlo = c->x0;
  const float xhi = c->x0 + c->knot_dx * (float)c->num_segments;
  const float x = fminf(fmaxf(s[0], xlo), xhi);
  int i = (int)floorf((x - xlo) / c->knot_dx);
  i = max(0, min(i, (int)c->num_segments - 1));
  const float sg = x - (xlo + c->knot_dx * (float)i);
  const float* k = c->coef[i];
  const float yc = k[0] + sg * (k[1] + sg * (k[2] + sg * k[3]));
  const float slope = k[1] + sg * (2.0f * k[2] + sg * 3.0f * k[3]);
  const float ey = s[1] - yc;
  const float eh = s[2] - atanf(slope);
  const float ev = s[3] - c->v_ref;
  return c->w_lat * ey * ey + c->w_head * eh * eh + c->w_speed * ev * ev;
}

__device__ float mppi_stage_cost(const float* s, const float* control,
                                 const uint8_t* model_params_raw, const uint8_t* cost_params_raw) {
  return bicycle_state_cost(s, reinterpret_cast<const BicycleCostParams*>(cost_params_raw));
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const BicycleCostParams* c = reinterpret_cast<const BicycleCostParams*>(cost_params_raw);
  return c->w_terminal * bicycle_state_cost(s, c);
}
