// wez_environment.cu — an ego vehicle driving to a goal among pursuing
// adversaries whose weapon-engagement zones switch on at random: the CUDA
// form of the reference's stochastic example plugin
// (examples/wez_environment_batch/wez_environment.metal:1-240), for its
// example application examples/wez_environment_batch/main.cpp.
//
// State (bytes, the example's AgentState): ego x, y, theta, v (floats),
// captured (bool at byte 16), then from byte 20 the adversaries, 20 bytes
// each: x, y, theta, v (floats), steps_since_active (uint16), active and
// terminal (bools).  The example's 8 adversaries make 180 bytes = 45 floats,
// more than the reference's 128-byte state buffer (its kernels truncate the
// state there); the library sizes the buffer from state_dim, and the
// adversary capacity here follows from it.
// Control: [acceleration, turn rate].
//
// Dynamics: the ego integrates a unicycle with acceleration (x, y from the
// previous heading and speed), wraps its heading to [-pi, pi) and clamps
// its speed to +-v_max.  An active adversary steers by pure pursuit toward the
// ego's new position (turn rate k * heading error), moves at constant speed,
// captures the ego inside the capture radius and retires after
// adv_max_steps.  An inactive, not yet retired adversary within
// adv_max_range of the ego activates with probability p: adv_fire_prob_max
// inside adv_min_range, falling linearly to 0 at adv_max_range.  The draw is
// the first word of Philox-2x32-10 at counter (c.x, c.y + 0x1000 + i) with
// the callable's counter c and key, so every adversary of every sample and
// step has its own stream (the reference's counter layout).
//
// Costs: stage = pos_weight |p - goal|^2 + control_weight |u|^2 + for every
// active adversary adv_collision_weight exp(-d^2 / (r_capture^2 + 1e-6));
// terminal = 10 pos_weight |p - goal|^2.
//
// Deviation from the reference: its cost callables read the adversaries
// through a view that starts them at byte 16 instead of 20
// (wez_environment.metal:59 vs :74), so its collision cost reads shifted
// fields; here both the dynamics and the costs read the adversaries where
// the state holds them.
#include "mppi_core.h"
#include "philox.h"
#include "model_params.h"

struct WezAdversary {
  float x, y, theta, v;
  uint16_t steps_since_active;
  bool active;
  bool terminal;
};

// Adversaries the state holds: (state bytes - 20) / 20.
#define MPPI_WEZ_CAPACITY ((MPPI_STATE_DIM * 4 - 20) / 20)
static_assert(MPPI_WEZ_CAPACITY >= 1, "the state holds no adversary");

struct WezState {
  float x, y, theta, v;
  bool captured;
  WezAdversary adv[MPPI_WEZ_CAPACITY];
};
static_assert(sizeof(WezAdversary) == 20, "adversary record is 20 bytes");
static_assert(sizeof(WezState) <= MPPI_STATE_DIM * 4, "state layout exceeds state_dim");

MPPI_PARAM_LAYOUT_OF(WezModelParams, WezCostParams, "mppi_b200/wez_environment/1")

#define MPPI_WEZ_PI 3.1415926535f

// x wrapped to [-pi, pi): fmod(x + pi, 2 pi), shifted into [0, 2 pi), - pi.
__device__ __forceinline__ float wez_wrap(float x) {
  float e = fmodf(x + MPPI_WEZ_PI, 2.0f * MPPI_WEZ_PI);
  if (e < 0.0f) e += 2.0f * MPPI_WEZ_PI;
  return e - MPPI_WEZ_PI;
}

__device__ __forceinline__ int wez_count(const WezModelParams* p) {
  return p->num_adversaries < MPPI_WEZ_CAPACITY ? p->num_adversaries : MPPI_WEZ_CAPACITY;
}

__device__ void mppi_dynamics(WezState* s, const float* control, const uint8_t* model_params_raw,
                              uint2 rng_counter, uint32_t rng_seed) {
  const WezModelParams* p = reinterpret_cast<const WezModelParams*>(model_params_raw);
  const float dt = p->dt;
  float sn, cs;
  mppi_sincosf(s->theta, &sn, &cs);
  const float v = s->v;
  s->x += v * cs * dt;
  s->y += v * sn * dt;
  s->theta += control[1] * dt;
  s->v += control[0] * dt;

  const int n = wez_count(p);
  for (int i = 0; i < n; ++i) {
    WezAdversary& a = s->adv[i];
    const float dx = s->x - a.x, dy = s->y - a.y;
    if (a.active) {
      const float target = atan2f(dy, dx);
      if (dx * dx + dy * dy < p->adv_capture_radius * p->adv_capture_radius) s->captured = true;
      const float omega = p->adv_k_gain * wez_wrap(target - a.theta);
      float as, ac;
      mppi_sincosf(a.theta, &as, &ac);
      a.x += a.v * ac * dt;
      a.y += a.v * as * dt;
      a.theta += omega * dt;
      a.steps_since_active = (uint16_t)(a.steps_since_active + 1);
      if ((int)a.steps_since_active > p->adv_max_steps) {
        a.active = false;
        a.terminal = true;
      }
    } else if (!a.terminal) {
      const float dist = sqrtf(dx * dx + dy * dy);
      if (dist < p->adv_max_range) {
        float prob = p->adv_fire_prob_max;
        if (dist > p->adv_min_range) {
          const float span = p->adv_max_range - p->adv_min_range;
          prob = span > 1e-6f ? prob * (p->adv_max_range - dist) / span : 0.0f;
        }
        const uint2 ctr = make_uint2(rng_counter.x, rng_counter.y + 0x1000u + (uint32_t)i);
        if (uint_to_01(philox2x32_10(ctr, rng_seed).x) < prob) {
          a.active = true;
          a.steps_since_active = 0;
        }
      }
    }
  }
  s->theta = wez_wrap(s->theta);
  s->v = fminf(fmaxf(s->v, -p->v_max), p->v_max);
}

__device__ float mppi_stage_cost(const WezState* s, const float* control,
                                 const uint8_t* model_params_raw, const uint8_t* cost_params_raw) {
  const WezModelParams* mp = reinterpret_cast<const WezModelParams*>(model_params_raw);
  const WezCostParams* c = reinterpret_cast<const WezCostParams*>(cost_params_raw);
  const float gx = s->x - c->x_goal, gy = s->y - c->y_goal;
  float cost = c->pos_weight * (gx * gx + gy * gy) +
               c->control_weight * (control[0] * control[0] + control[1] * control[1]);
  const float r2 = mp->adv_capture_radius * mp->adv_capture_radius + 1e-6f;
  const int n = wez_count(mp);
  for (int i = 0; i < n; ++i) {
    const WezAdversary& a = s->adv[i];
    if (a.active) {
      const float dx = s->x - a.x, dy = s->y - a.y;
      cost += c->adv_collision_weight * expf(-(dx * dx + dy * dy) / r2);
    }
  }
  return cost;
}

__device__ float mppi_terminal_cost(const WezState* s, const uint8_t* model_params_raw,
                                    const uint8_t* cost_params_raw) {
  const WezCostParams* c = reinterpret_cast<const WezCostParams*>(cost_params_raw);
  const float gx = s->x - c->x_goal, gy = s->y - c->y_goal;
  return c->pos_weight * (gx * gx + gy * gy) * 10.0f;
}
