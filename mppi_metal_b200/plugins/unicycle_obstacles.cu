// unicycle_obstacles.cu — kinematic unicycle among moving circular keep-out
// regions (layout and formulas in model_params.h).  State [x, y, theta, t],
// control [v, omega].
//
// The penetration max(0, r - |p - c(t)|) of every obstacle is evaluated
// branch-free (approximate square root), two obstacles per packed FP32x2
// instruction, in a loop unrolled to a compile-time bound chosen by one
// uniform branch on num_obs, so the obstacle pairs form independent
// instruction streams the compiler can interleave; the terms are summed as a
// tree.  The heading's sine and cosine
// come from the library's mppi_sincosf (about 1e-7 absolute).
//
// mppi_proposal_features gives the learned proposal its 31 inputs.
#include "mppi_core.h"
#include "model_params.h"

// The blobs this plugin reads (checked against the driver's ParamLayout).
MPPI_PARAM_LAYOUT_OF(UnicycleModelParams, UnicycleCostParams, "mppi_b200/unicycle_obstacles/1")

__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,
                              const uint8_t* model_params_raw, uint2 rng_counter,
                              uint32_t rng_seed) {
  const UnicycleModelParams* p = reinterpret_cast<const UnicycleModelParams*>(model_params_raw);
  float* s = reinterpret_cast<float*>(state_raw);
  const float dt = p->dt;
  float sn, cs;
  mppi_sincosf(s[2], &sn, &cs);
  s[0] += control[0] * cs * dt;
  s[1] += control[0] * sn * dt;
  s[2] += control[1] * dt;
  s[3] += dt;
}

__device__ __forceinline__ float unicycle_goal(const float* s, const UnicycleCostParams* c) {
  const float dx = s[0] - c->goal_x, dy = s[1] - c->goal_y;
  return c->w_goal * (dx * dx + dy * dy);
}

// Sum over obstacles [0, N) of max(0, r_i - |p - c_i(t)|), two obstacles per
// packed FP32x2 instruction (sm_100 FFMA2 / FADD2 / FMUL2, each lane rounded
// like the scalar operation, so the sum is the scalar loop's): the centre
// c = c0 + v t, the offset c - p, the squared distance, and the penetration
// as r - min(d, r).  MASK: obstacles at or beyond num_obs contribute nothing
// (not needed when num_obs == N).  The parameter arrays are 8-byte aligned
// in the blob, and the library passes blobs 16-byte aligned.
template <int N, bool MASK>
__device__ __forceinline__ float unicycle_penetration(const float* s, const UnicycleCostParams* c) {
  static_assert(N % 2 == 0, "obstacles come in pairs");
  const float t = s[3];
  const unsigned n = c->num_obs;
  const float2 tt = make_float2(t, t);
  const float2 nx = make_float2(-s[0], -s[0]), ny = make_float2(-s[1], -s[1]);
  const float2* cx2 = reinterpret_cast<const float2*>(c->obs_cx);
  const float2* cy2 = reinterpret_cast<const float2*>(c->obs_cy);
  const float2* vx2 = reinterpret_cast<const float2*>(c->obs_vx);
  const float2* vy2 = reinterpret_cast<const float2*>(c->obs_vy);
  const float2* r2 = reinterpret_cast<const float2*>(c->obs_r);
  float2 pen[N / 2];
#pragma unroll
  for (int j = 0; j < N / 2; ++j) {
    const float2 ex = __fadd2_rn(__ffma2_rn(vx2[j], tt, cx2[j]), nx);
    const float2 ey = __fadd2_rn(__ffma2_rn(vy2[j], tt, cy2[j]), ny);
    const float2 d2 = __ffma2_rn(ex, ex, __fmul2_rn(ey, ey));
    float2 r = r2[j];
    if (MASK) {
      r.x = (unsigned)(2 * j) < n ? r.x : 0.0f;
      r.y = (unsigned)(2 * j + 1) < n ? r.y : 0.0f;
    }
    const float2 m = make_float2(fminf(mppi_sqrt_approx(d2.x), r.x),
                                 fminf(mppi_sqrt_approx(d2.y), r.y));
    pen[j] = __fadd2_rn(r, make_float2(-m.x, -m.y));
  }
#pragma unroll
  for (int w = 1; w < N / 2; w *= 2)
#pragma unroll
    for (int i = 0; i + w < N / 2; i += 2 * w) pen[i] = __fadd2_rn(pen[i], pen[i + w]);
  return pen[0].x + pen[0].y;
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

// Part `part` of 4 of the stage cost, for the library's cooperative rollout
// (MPPI_STAGE_COST_SPLIT): the obstacle pairs [part * PP, (part + 1) * PP)
// with PP = num_obs / 8 pairs (1 for 8 obstacles, 2 for 16), and the goal
// term in part 0.  The four parts sum to mppi_stage_cost up to rounding.
template <int PP, bool MASK>
__device__ __forceinline__ float unicycle_penetration_part(const float* s,
                                                           const UnicycleCostParams* c,
                                                           int part) {
  const float t = s[3];
  const unsigned n = c->num_obs;
  const float2 tt = make_float2(t, t);
  const float2 nx = make_float2(-s[0], -s[0]), ny = make_float2(-s[1], -s[1]);
  const float2* cx2 = reinterpret_cast<const float2*>(c->obs_cx) + part * PP;
  const float2* cy2 = reinterpret_cast<const float2*>(c->obs_cy) + part * PP;
  const float2* vx2 = reinterpret_cast<const float2*>(c->obs_vx) + part * PP;
  const float2* vy2 = reinterpret_cast<const float2*>(c->obs_vy) + part * PP;
  const float2* r2 = reinterpret_cast<const float2*>(c->obs_r) + part * PP;
  float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int j = 0; j < PP; ++j) {
    const float2 ex = __fadd2_rn(__ffma2_rn(vx2[j], tt, cx2[j]), nx);
    const float2 ey = __fadd2_rn(__ffma2_rn(vy2[j], tt, cy2[j]), ny);
    const float2 d2 = __ffma2_rn(ex, ex, __fmul2_rn(ey, ey));
    float2 r = r2[j];
    if (MASK) {
      const unsigned i0 = (unsigned)(2 * (part * PP + j));
      r.x = i0 < n ? r.x : 0.0f;
      r.y = i0 + 1u < n ? r.y : 0.0f;
    }
    const float2 m = make_float2(fminf(mppi_sqrt_approx(d2.x), r.x),
                                 fminf(mppi_sqrt_approx(d2.y), r.y));
    acc = __fadd2_rn(acc, __fadd2_rn(r, make_float2(-m.x, -m.y)));
  }
  return acc.x + acc.y;
}

__device__ float mppi_stage_cost_part(const float* s, const float* control,
                                      const uint8_t* model_params_raw,
                                      const uint8_t* cost_params_raw, int part) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  const unsigned n = c->num_obs;
  float pen;
  if (n == MPPI_UNICYCLE_MAX_OBS)
    pen = unicycle_penetration_part<MPPI_UNICYCLE_MAX_OBS / 8, false>(s, c, part);
  else if (n == 8)
    pen = unicycle_penetration_part<1, false>(s, c, part);
  else if (n < 8)
    pen = unicycle_penetration_part<1, true>(s, c, part);
  else
    pen = unicycle_penetration_part<MPPI_UNICYCLE_MAX_OBS / 8, true>(s, c, part);
  const float goal = part == 0 ? unicycle_goal(s, c) : 0.0f;
  return fmaf(c->w_obs, pen, goal);
}

MPPI_STAGE_COST_SPLIT(mppi_stage_cost, mppi_stage_cost_part, 4)

__device__ float mppi_terminal_cost(const float* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  return c->w_terminal * unicycle_goal(s, c);
}

// Proposal features (31 of them):
//   [0..5)   x / 10, y / 10, cos(theta), sin(theta), t / 15
//   [5..7)   goal offset in the body frame (forward, left) / 10
//   [7..31)  the 8 obstacles of least clearance |p - c_i(t)| - r_i (ties:
//            lower index first), each as its centre's body-frame offset / 10
//            and its radius; missing obstacles give zeros
// The ranking is computed all at once: obstacle i's rank is the number of
// obstacles that come before it (smaller clearance, or equal clearance and
// lower index), 256 independent comparisons instead of eight dependent
// arg-min passes; the parameters are read into registers once.
__device__ void mppi_proposal_features(const float* s, const uint8_t* model_params_raw,
                                       const uint8_t* cost_params_raw, float* f) {
  const UnicycleCostParams* c = reinterpret_cast<const UnicycleCostParams*>(cost_params_raw);
  const float x = s[0], y = s[1], t = s[3];
  float sn, cs;
  mppi_sincosf(s[2], &sn, &cs);
  f[0] = x * 0.1f;
  f[1] = y * 0.1f;
  f[2] = cs;
  f[3] = sn;
  f[4] = t * (1.0f / 15.0f);
  const float gx = c->goal_x - x, gy = c->goal_y - y;
  f[5] = (cs * gx + sn * gy) * 0.1f;
  f[6] = (cs * gy - sn * gx) * 0.1f;
  const unsigned n = c->num_obs < MPPI_UNICYCLE_MAX_OBS ? c->num_obs : MPPI_UNICYCLE_MAX_OBS;
  const float inf = __int_as_float(0x7f800000);
  float ex[MPPI_UNICYCLE_MAX_OBS], ey[MPPI_UNICYCLE_MAX_OBS], clr[MPPI_UNICYCLE_MAX_OBS];
  float rad[MPPI_UNICYCLE_MAX_OBS];
#pragma unroll
  for (unsigned i = 0; i < MPPI_UNICYCLE_MAX_OBS; ++i) {
    rad[i] = c->obs_r[i];
    ex[i] = fmaf(c->obs_vx[i], t, c->obs_cx[i]) - x;
    ey[i] = fmaf(c->obs_vy[i], t, c->obs_cy[i]) - y;
    clr[i] = i < n ? sqrtf(ex[i] * ex[i] + ey[i] * ey[i]) - rad[i] : inf;
  }
#pragma unroll
  for (unsigned i = 0; i < MPPI_UNICYCLE_MAX_OBS; ++i) {
    unsigned rank = 0;
#pragma unroll
    for (unsigned j = 0; j < MPPI_UNICYCLE_MAX_OBS; ++j)
      rank += (clr[j] < clr[i] || (j < i && clr[j] == clr[i])) ? 1u : 0u;
    if (i < n && rank < 8) {
      f[7 + 3 * rank] = (cs * ex[i] + sn * ey[i]) * 0.1f;
      f[8 + 3 * rank] = (cs * ey[i] - sn * ex[i]) * 0.1f;
      f[9 + 3 * rank] = rad[i];
    }
  }
}
