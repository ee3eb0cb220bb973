// gust_integrator.cu — a stochastic model: the dynamics draw their own
// randoms from the counter and key the library passes in (layout and
// formulas in model_params.h).  Written with the reference's helper names
// (philox2x32_10, uint_to_01, box_muller), as a plugin for the reference
// would be.
#include "mppi_core.h"
#include "philox.h"
#include "model_params.h"

// The blob this plugin reads (no cost parameters), checked against the
// driver's ParamLayout.
MPPI_PARAM_LAYOUT(sizeof(GustModelParams), alignof(GustModelParams), 0, 1,
                  "mppi_b200/gust_integrator/1")

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const GustModelParams* p = reinterpret_cast<const GustModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float2 n = box_muller(philox2x32_10(rng_counter, rng_seed));
  const uint2 ev = make_uint2(rng_counter.x, rng_counter.y + 0x1000u);
  if (uint_to_01(philox2x32_10(ev, rng_seed).x) < p->p_event) s[4] = 1.0f;
  const float dt = p->dt;
  s[2] += (control[0] + p->noise_std * n.x + s[4] * p->gust_accel) * dt;
  s[3] += (control[1] + p->noise_std * n.y) * dt;
  s[0] += s[2] * dt;
  s[1] += s[3] * dt;
}

__device__ float mppi_stage_cost(const float* s, const float* control,
                                 const uint8_t* model_params, const uint8_t* cost_params) {
  return s[0] * s[0] + s[1] * s[1] + 0.1f * (s[2] * s[2] + s[3] * s[3]);
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params,
                                    const uint8_t* cost_params) {
  return 10.0f * (s[0] * s[0] + s[1] * s[1]);
}
