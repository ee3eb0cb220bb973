// quadrotor.cu — 12-state rigid-body quadrotor with four rotor thrusts
// (layout and formulas in model_params.h).  State [p(3), v(3), phi, theta,
// psi, p, q, r], control [f1..f4].  Cost: waypoint tracking plus the
// penetration of up to 32 spherical obstacles, evaluated branch-free.
#include "mppi_core.h"
#include "model_params.h"

__device__ void mppi_dynamics(uint8_t* state_raw, const float* u,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const QuadrotorModelParams* mp = reinterpret_cast<const QuadrotorModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = mp->dt;
  const float vx = s[3], vy = s[4], vz = s[5];
  const float ph = s[6], th = s[7], ps = s[8];
  const float p = s[9], q = s[10], r = s[11];
  const float T = u[0] + u[1] + u[2] + u[3];
  const float tx = mp->arm * (u[1] - u[3]);
  const float ty = mp->arm * (u[2] - u[0]);
  const float tz = mp->yaw_coef * (u[0] - u[1] + u[2] - u[3]);
  float sph, cph, sth, cth, sps, cps;
  sincosf(ph, &sph, &cph);
  sincosf(th, &sth, &cth);
  sincosf(ps, &sps, &cps);
  const float zx = cph * sth * cps + sph * sps;
  const float zy = cph * sth * sps - sph * cps;
  const float zz = cph * cth;
  const float a = T / mp->mass;
  const float qs = q * sph + r * cph;
  const float dph = p + qs * (sth / cth);
  const float dth = q * cph - r * sph;
  const float dps = qs / cth;
  const float dp = (tx - (mp->jz - mp->jy) * q * r) / mp->jx;
  const float dq = (ty - (mp->jx - mp->jz) * r * p) / mp->jy;
  const float dr = (tz - (mp->jy - mp->jx) * p * q) / mp->jz;
  s[0] += vx * dt;
  s[1] += vy * dt;
  s[2] += vz * dt;
  s[3] += a * zx * dt;
  s[4] += a * zy * dt;
  s[5] += (a * zz - mp->gravity) * dt;
  s[6] += dph * dt;
  s[7] += dth * dt;
  s[8] += dps * dt;
  s[9] += dp * dt;
  s[10] += dq * dt;
  s[11] += dr * dt;
}

__device__ __forceinline__ float quad_position_cost(const float* s, const QuadrotorCostParams* c) {
  const float dx = s[0] - c->wp_x, dy = s[1] - c->wp_y, dz = s[2] - c->wp_z;
  return c->w_pos * (dx * dx + dy * dy + dz * dz);
}

__device__ float mppi_stage_cost(const float* s, const float* u, const uint8_t* model_params_raw,
                                 const uint8_t* cost_params_raw) {
  const QuadrotorCostParams* c = reinterpret_cast<const QuadrotorCostParams*>(cost_params_raw);
  const unsigned n = c->num_obs;
  float pen[MPPI_QUAD_MAX_OBS];
#pragma unroll
  for (int i = 0; i < MPPI_QUAD_MAX_OBS; ++i) {
    const float ex = s[0] - c->obs_cx[i], ey = s[1] - c->obs_cy[i], ez = s[2] - c->obs_cz[i];
    const float d = mppi_sqrt_approx(fmaf(ex, ex, fmaf(ey, ey, ez * ez)));
    const float rad = (unsigned)i < n ? c->obs_r[i] : 0.0f;
    pen[i] = fmaxf(rad - d, 0.0f);
  }
#pragma unroll
  for (int w = 1; w < MPPI_QUAD_MAX_OBS; w *= 2)
#pragma unroll
    for (int i = 0; i + w < MPPI_QUAD_MAX_OBS; i += 2 * w) pen[i] += pen[i + w];
  const float vel = c->w_vel * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  const float att = c->w_att * (s[6] * s[6] + s[7] * s[7]);
  const float rate = c->w_rate * (s[9] * s[9] + s[10] * s[10] + s[11] * s[11]);
  return quad_position_cost(s, c) + vel + att + rate + c->w_obs * pen[0];
}

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const QuadrotorCostParams* c = reinterpret_cast<const QuadrotorCostParams*>(cost_params_raw);
  return c->w_terminal * quad_position_cost(s, c);
}
