// unicycle_obstacles.cu — kinematic unicycle among moving circular keep-out
// regions (layout and formulas in model_params.h).  State [x, y, theta, t],
// control [v, omega].
//
// The penetration max(0, r - |p - c(t)|) of every obstacle is evaluated
// branch-free (approximate square root), in a loop unrolled to a
// compile-time bound chosen by one uniform branch on num_obs, so the
// obstacles form independent instruction streams the compiler can
// interleave; the terms are summed as a tree.
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

// Sum over obstacles [0, N) of max(0, r_i - |p - c_i(t)|).  MASK: obstacles
// at or beyond num_obs contribute nothing (not needed when num_obs == N).
template <int N, bool MASK>
__device__ __forceinline__ float unicycle_penetration(const float* s, const UnicycleCostParams* c) {
  const float t = s[3];
  const unsigned n = c->num_obs;
  float pen[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const float cx = fmaf(c->obs_vx[i], t, c->obs_cx[i]);
    const float cy = fmaf(c->obs_vy[i], t, c->obs_cy[i]);
    const float ex = s[0] - cx, ey = s[1] - cy;
    const float d = mppi_sqrt_approx(fmaf(ex, ex, ey * ey));
    const float r = (!MASK || (unsigned)i < n) ? c->obs_r[i] : 0.0f;
    pen[i] = fmaxf(r - d, 0.0f);
  }
#pragma unroll
  for (int w = 1; w < N; w *= 2)
#pragma unroll
    for (int i = 0; i + w < N; i += 2 * w) pen[i] += pen[i + w];
  return pen[0];
}

__device__ float mppi_stage_cost(const float* s, const float* control,
                                 const uint8_t* model_params_raw, const uint8_t* cost_params_raw) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  const unsigned n = c->num_obs;
  float pen;
  if (n == MPPI_UNICYCLE_MAX_OBS)
    pen = unicycle_penetration<MPPI_UNICYCLE_MAX_OBS, false>(s, c);
  else if (n == 8)
    pen = unicycle_penetration<8, false>(s, c);
  else if (n < 8)
    pen = unicycle_penetration<8, true>(s, c);
  else
    pen = unicycle_penetration<MPPI_UNICYCLE_MAX_OBS, true>(s, c);
  return unicycle_goal(s, c) + c->w_obs * pen;
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  return c->w_terminal * unicycle_goal(s, c);
}
