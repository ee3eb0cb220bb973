// quadrotor.cu — 12-state rigid-body quadrotor with four rotor thrusts
// (layout and formulas in model_params.h).  State [p(3), v(3), phi, theta,
// psi, p, q, r], control [f1..f4].  Cost: waypoint tracking plus the
// penetration of up to 32 spherical obstacles, evaluated branch-free.
// mppi_proposal_features gives the learned proposal its 29 inputs.
#include "mppi_core.h"
#include "model_params.h"

// The blobs this plugin reads (checked against the driver's ParamLayout).
MPPI_PARAM_LAYOUT_OF(QuadrotorModelParams, QuadrotorCostParams, "mppi_b200/quadrotor/1")

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
  mppi_sincosf(ph, &sph, &cph);
  mppi_sincosf(th, &sth, &cth);
  mppi_sincosf(ps, &sps, &cps);
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

// Proposal features (29 of them):
//   [0..3)   (p - waypoint) / 4        [3..6)   v / 2
//   [6..9)   phi, theta, psi           [9..12)  body rates / 4
//   [12]     z / 4
//   [13..29) the 4 obstacles of least clearance |p - c_i| - r_i (ties: lower
//            index first): (c_i - p) / 4 and r_i; missing ones give zeros
// The ranking stays in registers (4 unrolled arg-min passes over 32 slots).
__device__ void mppi_proposal_features(const float* s, const uint8_t* model_params_raw,
                                       const uint8_t* cost_params_raw, float* f) {
  const QuadrotorCostParams* c = reinterpret_cast<const QuadrotorCostParams*>(cost_params_raw);
  f[0] = (s[0] - c->wp_x) * 0.25f;
  f[1] = (s[1] - c->wp_y) * 0.25f;
  f[2] = (s[2] - c->wp_z) * 0.25f;
  f[3] = s[3] * 0.5f;
  f[4] = s[4] * 0.5f;
  f[5] = s[5] * 0.5f;
  f[6] = s[6];
  f[7] = s[7];
  f[8] = s[8];
  f[9] = s[9] * 0.25f;
  f[10] = s[10] * 0.25f;
  f[11] = s[11] * 0.25f;
  f[12] = s[2] * 0.25f;
  const unsigned n = c->num_obs < MPPI_QUAD_MAX_OBS ? c->num_obs : MPPI_QUAD_MAX_OBS;
  const float inf = __int_as_float(0x7f800000);
  float clr[MPPI_QUAD_MAX_OBS];
#pragma unroll
  for (unsigned i = 0; i < MPPI_QUAD_MAX_OBS; ++i) {
    const float ex = c->obs_cx[i] - s[0], ey = c->obs_cy[i] - s[1], ez = c->obs_cz[i] - s[2];
    clr[i] = i < n ? sqrtf(ex * ex + ey * ey + ez * ez) - c->obs_r[i] : inf;
  }
#pragma unroll
  for (unsigned j = 0; j < 4; ++j) {
    float bv = inf;
    unsigned best = MPPI_QUAD_MAX_OBS;
#pragma unroll
    for (unsigned i = 0; i < MPPI_QUAD_MAX_OBS; ++i) {
      const bool take = clr[i] < bv;  // strict: the lower index wins ties
      bv = take ? clr[i] : bv;
      best = take ? i : best;
    }
#pragma unroll
    for (unsigned i = 0; i < MPPI_QUAD_MAX_OBS; ++i) clr[i] = i == best ? inf : clr[i];
    if (best < MPPI_QUAD_MAX_OBS) {
      f[13 + 4 * j] = (c->obs_cx[best] - s[0]) * 0.25f;
      f[14 + 4 * j] = (c->obs_cy[best] - s[1]) * 0.25f;
      f[15 + 4 * j] = (c->obs_cz[best] - s[2]) * 0.25f;
      f[16 + 4 * j] = c->obs_r[best];
    }
  }
}
