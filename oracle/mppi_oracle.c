/*
 * mppi_oracle.c — FP64 CPU restatement of the reference MPPI hot path.
 * TEST INFRASTRUCTURE ONLY (see mppi_oracle.h for scope and citations).
 */
#include "mppi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "../mppi_metal_b200/plugins/model_params.h"

#define MAX_STATE 128 /* the library's state limit (MPPI_MAX_STATE_DIM floats) */
#define ORACLE_PI 3.14159265358979323846
#define MAX_CTRL 16

/* ---- Philox-2x32-10 (shaders/philox.h:19-36) ---------------------------- */
/* Round: 32x32->64 product of the first word with 0xD256D193; the new first
 * word is hi ^ key ^ second word, the new second word is lo; the key is
 * bumped by the Weyl constant 0x9E3779B9 after every round. */
void oracle_philox2x32_10(uint32_t c0, uint32_t c1, uint32_t key, uint32_t out[2]) {
  for (int i = 0; i < 10; ++i) {
    const uint64_t prod = (uint64_t)c0 * 0xD256D193u;
    const uint32_t hi = (uint32_t)(prod >> 32);
    const uint32_t lo = (uint32_t)prod;
    c0 = hi ^ key ^ c1;
    c1 = lo;
    key += 0x9E3779B9u;
  }
  out[0] = c0;
  out[1] = c1;
}

void oracle_philox_many(uint64_t n, const uint32_t* c0, const uint32_t* c1,
                        const uint32_t* key, uint32_t* out) {
  for (uint64_t i = 0; i < n; ++i) oracle_philox2x32_10(c0[i], c1[i], key[i], out + 2 * i);
}

/* shaders/philox.h:39-41: (float(x) + 0.5f) * (1/2^32), two float ops. */
float oracle_uint_to_01(uint32_t x) {
  volatile float f = (float)x; /* round-to-nearest int -> float */
  volatile float s = f + 0.5f;
  return s * (1.0f / 4294967296.0f);
}

/* shaders/philox.h:44-50: r = sqrt(-2 ln u1), theta = 2 pi u2. */
void oracle_box_muller(uint32_t w0, uint32_t w1, double out[2]) {
  const double u1 = (double)oracle_uint_to_01(w0);
  const double u2 = (double)oracle_uint_to_01(w1);
  const double r = sqrt(-2.0 * log(u1));
  const double th = 2.0 * ORACLE_PI * u2;
  out[0] = r * cos(th);
  out[1] = r * sin(th);
}

int oracle_cholesky(uint32_t m, const double* a, double* l) {
  memset(l, 0, sizeof(double) * m * m);
  for (uint32_t i = 0; i < m; ++i) {
    for (uint32_t j = 0; j <= i; ++j) {
      double s = a[i * m + j];
      for (uint32_t k = 0; k < j; ++k) s -= l[i * m + k] * l[j * m + k];
      if (i == j) {
        if (s <= 0.0) return -1;
        l[i * m + i] = sqrt(s);
      } else {
        l[i * m + j] = s / l[j * m + j];
      }
    }
  }
  return 0;
}

/* Noise for sample k at every time step.  Counter layout
 * (shaders/mppi_rollout.metal:66,73-87; mppi_reduce.metal:151-162):
 *   ctr = (step, k*H*P + t*P + d/2), P = ceil(m/2), key = agent key;
 *   the pair's first normal goes to dim d (even), the second to d+1.
 * Shaping: diagonal eps_d = n_d * sigma_d (sigma = std-dev); full covariance
 * eps = L n with L the Cholesky factor of sigma (project extension).
 * Half-precision noise modes with m >= 3 (project extension, the device's
 * mppi_box_muller_fast16): ctr = (step, k*H*Q + t*Q + q), Q = ceil(m/4); each
 * 32-bit word gives two 16-bit uniforms u = (h + 1/2) / 65536 (lower half
 * u1, upper u2) and one Box-Muller pair: word x dims 4q, 4q+1, word y dims
 * 4q+2, 4q+3; the shaped value is rounded to binary16. */
void oracle_sample_noise(const oracle_problem* p, uint32_t step, uint32_t key,
                         uint32_t k, const double* sigma, double* normals,
                         double* eps) {
  const uint32_t H = p->horizon, m = p->control_dim, P = (m + 1) / 2;
  double L[MAX_CTRL * MAX_CTRL];
  if (p->cov_full) oracle_cholesky(m, sigma, L);
  const int noise16 = p->noise_half && m >= 3; /* four 16-bit uniforms per call */
  const uint32_t Q = (m + 3) / 4;
  for (uint32_t t = 0; t < H; ++t) {
    double n[MAX_CTRL + 4];
    for (uint32_t q = 0; noise16 && q < Q; ++q) {
      const uint32_t c1 = k * H * Q + t * Q + q; /* uint32 wrap as on the device */
      uint32_t w[2];
      oracle_philox2x32_10(step, c1, key, w);
      for (int h = 0; h < 2; ++h) {
        const double u1 = ((double)(w[h] & 0xffffu) + 0.5) / 65536.0;
        const double u2 = ((double)(w[h] >> 16) + 0.5) / 65536.0;
        const double r = sqrt(-2.0 * log(u1));
        n[4 * q + 2 * h] = r * cos(2.0 * ORACLE_PI * u2);
        n[4 * q + 2 * h + 1] = r * sin(2.0 * ORACLE_PI * u2);
      }
    }
    for (uint32_t d = 0; !noise16 && d < m; d += 2) {
      const uint32_t pair = t * P + d / 2;
      const uint32_t c1 = k * H * P + pair; /* uint32 wrap as on the device */
      uint32_t w[2];
      double g[2];
      oracle_philox2x32_10(step, c1, key, w);
      oracle_box_muller(w[0], w[1], g);
      n[d] = g[0];
      if (d + 1 < m) n[d + 1] = g[1];
    }
    for (uint32_t d = 0; d < m; ++d) {
      if (normals) normals[t * m + d] = n[d];
      if (eps) {
        double e;
        if (p->cov_full) {
          e = 0.0;
          for (uint32_t j = 0; j <= d; ++j) e += L[d * m + j] * n[j];
        } else {
          e = n[d] * sigma[d];
        }
        if (p->noise_half) e = (double)(_Float16)(float)e; /* round to binary16 */
        eps[t * m + d] = e;
      }
    }
  }
}

/* ---- model restatements ------------------------------------------------- */

static void dyn_double_integrator(double* s, const double* u) {
  /* shaders/test_user_dynamics.metal:8-19 */
  const double dt = (double)0.1f;
  s[0] += s[2] * dt;
  s[1] += s[3] * dt;
  s[2] += u[0] * dt;
  s[3] += u[1] * dt;
}

static void dyn_nonholonomic(double* s, const double* u, const NonholonomicModelParams* mp) {
  /* examples/nonholonomic_vehicle/nonholonomic_vehicle.metal:24-55 */
  const double dt = mp->dt;
  const double th = s[2], v = s[3];
  s[0] += v * cos(th) * dt;
  s[1] += v * sin(th) * dt;
  s[2] += u[1] * dt;
  s[3] += u[0] * dt;
  const double pi = (double)3.1415926535f;
  s[2] = fmod(s[2] + pi, 2.0 * pi);
  if (s[2] < 0) s[2] += 2.0 * pi;
  s[2] -= pi;
  if (s[3] > mp->v_max) s[3] = mp->v_max;
  if (s[3] < -mp->v_max) s[3] = -mp->v_max;
}

static void dyn_unicycle(double* s, const double* u, const UnicycleModelParams* mp) {
  const double dt = mp->dt;
  const double th = s[2];
  s[0] += u[0] * cos(th) * dt;
  s[1] += u[0] * sin(th) * dt;
  s[2] += u[1] * dt;
  s[3] += dt;
}

static void dyn_bicycle(double* s, const double* u, const BicycleModelParams* mp) {
  const double dt = mp->dt;
  const double th = s[2], v = s[3], de = s[4];
  s[0] += v * cos(th) * dt;
  s[1] += v * sin(th) * dt;
  s[2] += v / mp->wheelbase * tan(de) * dt;
  s[3] += u[0] * dt;
  double nd = de + u[1] * dt;
  if (nd > mp->delta_max) nd = mp->delta_max;
  if (nd < -mp->delta_max) nd = -mp->delta_max;
  s[4] = nd;
}

static void dyn_quadrotor(double* s, const double* u, const QuadrotorModelParams* mp) {
  const double dt = mp->dt;
  const double vx = s[3], vy = s[4], vz = s[5];
  const double ph = s[6], th = s[7];
  const double p = s[9], q = s[10], r = s[11];
  const double f1 = u[0], f2 = u[1], f3 = u[2], f4 = u[3];
  const double T = f1 + f2 + f3 + f4;
  const double tx = mp->arm * (f2 - f4);
  const double ty = mp->arm * (f3 - f1);
  const double tz = mp->yaw_coef * (f1 - f2 + f3 - f4);
  const double cph = cos(ph), sph = sin(ph), cth = cos(th), sth = sin(th);
  const double cps = cos(s[8]), sps = sin(s[8]);
  const double zx = cph * sth * cps + sph * sps;
  const double zy = cph * sth * sps - sph * cps;
  const double zz = cph * cth;
  const double a = T / mp->mass;
  const double ax = a * zx, ay = a * zy, az = a * zz - mp->gravity;
  const double tth = sth / cth;
  const double dph = p + (q * sph + r * cph) * tth;
  const double dth = q * cph - r * sph;
  const double dps = (q * sph + r * cph) / cth;
  const double dp = (tx - (mp->jz - mp->jy) * q * r) / mp->jx;
  const double dq = (ty - (mp->jx - mp->jz) * r * p) / mp->jy;
  const double dr = (tz - (mp->jy - mp->jx) * p * q) / mp->jz;
  s[0] += vx * dt;
  s[1] += vy * dt;
  s[2] += vz * dt;
  s[3] += ax * dt;
  s[4] += ay * dt;
  s[5] += az * dt;
  s[6] += dph * dt;
  s[7] += dth * dt;
  s[8] += dps * dt;
  s[9] += dp * dt;
  s[10] += dq * dt;
  s[11] += dr * dt;
}

/* gust_integrator (plugins/gust_integrator.cu): stochastic dynamics drawing
 * from the callable's counter and key; the event test compares the
 * bit-exact float uniform, so both sides take the same branch. */
static void dyn_gust(double* s, const double* u, const GustModelParams* mp, uint32_t ctr0,
                     uint32_t ctr1, uint32_t key) {
  uint32_t w[2], e[2];
  double n[2];
  oracle_philox2x32_10(ctr0, ctr1, key, w);
  oracle_box_muller(w[0], w[1], n);
  oracle_philox2x32_10(ctr0, ctr1 + 0x1000u, key, e);
  if (oracle_uint_to_01(e[0]) < mp->p_event) s[4] = 1.0;
  const double dt = mp->dt;
  s[2] += (u[0] + (double)mp->noise_std * n[0] + s[4] * (double)mp->gust_accel) * dt;
  s[3] += (u[1] + (double)mp->noise_std * n[1]) * dt;
  s[0] += s[2] * dt;
  s[1] += s[3] * dt;
}

/* wez_environment (plugins/wez_environment.cu), following the reference's
 * examples/wez_environment_batch/wez_environment.metal:84-184 (dynamics) and
 * :186-240 (costs), with the adversaries read where the state holds them
 * (the reference's cost view starts them 4 bytes early, :59 vs :74).
 * State slots (the example's AgentState as floats): [0, 4) ego x, y, theta,
 * v; [4] a packed word (byte 0: captured); adversary i at 5 + 5 i: x, y,
 * theta, v and a packed word (bytes 0-1 steps_since_active, byte 2 active,
 * byte 3 terminal).  A packed word travels as the float with its bits; a
 * float converts to double and back exactly, so the bits survive.  The
 * activation draw compares the bit-exact float uniform. */
static uint32_t wez_bits(double v) {
  const float f = (float)v;
  uint32_t b;
  memcpy(&b, &f, 4);
  return b;
}
static double wez_from_bits(uint32_t b) {
  float f;
  memcpy(&f, &b, 4);
  return (double)f;
}
static double wez_wrap(double x) {
  const double pi = (double)3.1415926535f;
  double e = fmod(x + pi, 2.0 * pi);
  if (e < 0.0) e += 2.0 * pi;
  return e - pi;
}
static int wez_count(const oracle_problem* p, const WezModelParams* mp) {
  const int cap = ((int)p->state_dim * 4 - 20) / 20;
  return mp->num_adversaries < cap ? mp->num_adversaries : cap;
}

static void dyn_wez(const oracle_problem* p, double* s, const double* u,
                    const WezModelParams* mp, uint32_t ctr0, uint32_t ctr1, uint32_t key) {
  const double dt = mp->dt;
  const double th = s[2], v = s[3];
  s[0] += v * cos(th) * dt;
  s[1] += v * sin(th) * dt;
  s[2] += u[1] * dt;
  s[3] += u[0] * dt;
  uint32_t ego = wez_bits(s[4]);
  const int n = wez_count(p, mp);
  for (int i = 0; i < n; ++i) {
    double* a = s + 5 + 5 * i;
    uint32_t w = wez_bits(a[4]);
    uint32_t steps = w & 0xffffu;
    int active = (w >> 16) & 0xffu, terminal = (w >> 24) & 0xffu;
    const double dx = s[0] - a[0], dy = s[1] - a[1];
    if (active) {
      const double target = atan2(dy, dx);
      const double rc = mp->adv_capture_radius;
      if (dx * dx + dy * dy < rc * rc) ego = (ego & ~0xffu) | 1u;
      const double omega = mp->adv_k_gain * wez_wrap(target - a[2]);
      a[0] += a[3] * cos(a[2]) * dt;
      a[1] += a[3] * sin(a[2]) * dt;
      a[2] += omega * dt;
      steps = (steps + 1u) & 0xffffu;
      if ((int)steps > mp->adv_max_steps) {
        active = 0;
        terminal = 1;
      }
    } else if (!terminal) {
      const double dist = sqrt(dx * dx + dy * dy);
      if (dist < mp->adv_max_range) {
        double prob = mp->adv_fire_prob_max;
        if (dist > mp->adv_min_range) {
          const double span = (double)mp->adv_max_range - mp->adv_min_range;
          prob = span > (double)1e-6f ? prob * (mp->adv_max_range - dist) / span : 0.0;
        }
        uint32_t r[2];
        oracle_philox2x32_10(ctr0, ctr1 + 0x1000u + (uint32_t)i, key, r);
        if ((double)oracle_uint_to_01(r[0]) < prob) {
          active = 1;
          steps = 0;
        }
      }
    }
    a[4] = wez_from_bits(steps | ((uint32_t)active << 16) | ((uint32_t)terminal << 24));
  }
  s[4] = wez_from_bits(ego);
  s[2] = wez_wrap(s[2]);
  if (s[3] > mp->v_max) s[3] = mp->v_max;
  if (s[3] < -mp->v_max) s[3] = -mp->v_max;
}

static double wez_stage_cost(const oracle_problem* p, const double* s, const double* u,
                             const WezModelParams* mp, const WezCostParams* cp) {
  const double gx = s[0] - cp->x_goal, gy = s[1] - cp->y_goal;
  double c = cp->pos_weight * (gx * gx + gy * gy) +
             cp->control_weight * (u[0] * u[0] + u[1] * u[1]);
  const double r2 = (double)mp->adv_capture_radius * mp->adv_capture_radius + (double)1e-6f;
  const int n = wez_count(p, mp);
  for (int i = 0; i < n; ++i) {
    const double* a = s + 5 + 5 * i;
    if ((wez_bits(a[4]) >> 16) & 0xffu) {
      const double dx = s[0] - a[0], dy = s[1] - a[1];
      c += cp->adv_collision_weight * exp(-(dx * dx + dy * dy) / r2);
    }
  }
  return c;
}

void oracle_dynamics(const oracle_problem* p, double* x, const double* u,
                     const void* model_params, uint32_t ctr0, uint32_t ctr1,
                     uint32_t key) {
  switch (p->model) {
    case ORACLE_MODEL_GUST:
      dyn_gust(x, u, (const GustModelParams*)model_params, ctr0, ctr1, key);
      break;
    case ORACLE_MODEL_WEZ:
      dyn_wez(p, x, u, (const WezModelParams*)model_params, ctr0, ctr1, key);
      break;
    case ORACLE_MODEL_DOUBLE_INTEGRATOR: dyn_double_integrator(x, u); break;
    case ORACLE_MODEL_NONHOLONOMIC:
      dyn_nonholonomic(x, u, (const NonholonomicModelParams*)model_params);
      break;
    case ORACLE_MODEL_UNICYCLE_OBSTACLES:
      dyn_unicycle(x, u, (const UnicycleModelParams*)model_params);
      break;
    case ORACLE_MODEL_BICYCLE_LANE:
      dyn_bicycle(x, u, (const BicycleModelParams*)model_params);
      break;
    case ORACLE_MODEL_QUADROTOR:
      dyn_quadrotor(x, u, (const QuadrotorModelParams*)model_params);
      break;
    default: break;
  }
}

static double unicycle_state_cost(const double* s, const UnicycleCostParams* cp, int terminal) {
  const double dx = s[0] - cp->goal_x, dy = s[1] - cp->goal_y;
  const double g = cp->w_goal * (dx * dx + dy * dy);
  if (terminal) return cp->w_terminal * g;
  double pen = 0.0;
  const double t = s[3];
  for (uint32_t i = 0; i < cp->num_obs && i < MPPI_UNICYCLE_MAX_OBS; ++i) {
    const double cx = cp->obs_cx[i] + cp->obs_vx[i] * t;
    const double cy = cp->obs_cy[i] + cp->obs_vy[i] * t;
    const double ex = s[0] - cx, ey = s[1] - cy;
    const double d = sqrt(ex * ex + ey * ey);
    const double v = cp->obs_r[i] - d;
    if (v > 0.0) pen += v;
  }
  return g + cp->w_obs * pen;
}

static double bicycle_state_cost(const double* s, const BicycleCostParams* cp) {
  const double xlo = cp->x0;
  const double xhi = cp->x0 + cp->knot_dx * cp->num_segments;
  double x = s[0];
  if (x < xlo) x = xlo;
  if (x > xhi) x = xhi;
  int i = (int)floor((x - xlo) / cp->knot_dx);
  if (i < 0) i = 0;
  if (i > (int)cp->num_segments - 1) i = (int)cp->num_segments - 1;
  const double sg = x - (xlo + cp->knot_dx * i);
  const float* c = cp->coef[i];
  const double yc = c[0] + sg * (c[1] + sg * (c[2] + sg * c[3]));
  const double slope = c[1] + sg * (2.0 * c[2] + sg * 3.0 * c[3]);
  const double ey = s[1] - yc;
  const double eh = s[2] - atan(slope);
  const double ev = s[3] - cp->v_ref;
  return cp->w_lat * ey * ey + cp->w_head * eh * eh + cp->w_speed * ev * ev;
}

static double quad_state_cost(const double* s, const QuadrotorCostParams* cp, int terminal) {
  const double dx = s[0] - cp->wp_x, dy = s[1] - cp->wp_y, dz = s[2] - cp->wp_z;
  const double pos = cp->w_pos * (dx * dx + dy * dy + dz * dz);
  if (terminal) return cp->w_terminal * pos;
  const double vel = cp->w_vel * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]);
  const double att = cp->w_att * (s[6] * s[6] + s[7] * s[7]);
  const double rate = cp->w_rate * (s[9] * s[9] + s[10] * s[10] + s[11] * s[11]);
  double pen = 0.0;
  for (uint32_t i = 0; i < cp->num_obs && i < MPPI_QUAD_MAX_OBS; ++i) {
    const double ex = s[0] - cp->obs_cx[i], ey = s[1] - cp->obs_cy[i], ez = s[2] - cp->obs_cz[i];
    const double v = cp->obs_r[i] - sqrt(ex * ex + ey * ey + ez * ez);
    if (v > 0.0) pen += v;
  }
  return pos + vel + att + rate + cp->w_obs * pen;
}

double oracle_stage_cost(const oracle_problem* p, const double* x, const double* u,
                         const void* model_params, const void* cost_params) {
  (void)model_params;
  if (!p->use_stage) return 0.0; /* shaders/mppi_rollout.metal:11-18 */
  switch (p->model) {
    case ORACLE_MODEL_DOUBLE_INTEGRATOR:
      return x[0] * x[0] + x[1] * x[1]; /* test_user_dynamics.metal:22-31 */
    case ORACLE_MODEL_NONHOLONOMIC: {
      /* nonholonomic_vehicle.metal:57-77 */
      const NonholonomicCostParams* cp = (const NonholonomicCostParams*)cost_params;
      const double dx = x[0] - cp->x_goal, dy = x[1] - cp->y_goal;
      double c = cp->pos_weight * (dx * dx + dy * dy);
      c += cp->control_weight * (u[0] * u[0] + u[1] * u[1]);
      return c;
    }
    case ORACLE_MODEL_UNICYCLE_OBSTACLES:
      return unicycle_state_cost(x, (const UnicycleCostParams*)cost_params, 0);
    case ORACLE_MODEL_BICYCLE_LANE:
      return bicycle_state_cost(x, (const BicycleCostParams*)cost_params);
    case ORACLE_MODEL_QUADROTOR:
      return quad_state_cost(x, (const QuadrotorCostParams*)cost_params, 0);
    case ORACLE_MODEL_GUST: /* plugins/gust_integrator.cu */
      return x[0] * x[0] + x[1] * x[1] + (double)0.1f * (x[2] * x[2] + x[3] * x[3]);
    case ORACLE_MODEL_WEZ:
      return wez_stage_cost(p, x, u, (const WezModelParams*)model_params,
                            (const WezCostParams*)cost_params);
    default: return 0.0;
  }
}

double oracle_terminal_cost(const oracle_problem* p, const double* x,
                            const void* model_params, const void* cost_params) {
  (void)model_params;
  if (!p->use_terminal) return 0.0; /* shaders/mppi_rollout.metal:20-28 */
  switch (p->model) {
    case ORACLE_MODEL_DOUBLE_INTEGRATOR:
      return x[0] * x[0] + x[1] * x[1]; /* test_user_dynamics.metal:33-43 */
    case ORACLE_MODEL_NONHOLONOMIC: {
      const NonholonomicCostParams* cp = (const NonholonomicCostParams*)cost_params;
      const double dx = x[0] - cp->x_goal, dy = x[1] - cp->y_goal;
      return cp->pos_weight * (dx * dx + dy * dy) * 10.0; /* :79-91 */
    }
    case ORACLE_MODEL_UNICYCLE_OBSTACLES:
      return unicycle_state_cost(x, (const UnicycleCostParams*)cost_params, 1);
    case ORACLE_MODEL_BICYCLE_LANE: {
      const BicycleCostParams* cp = (const BicycleCostParams*)cost_params;
      return cp->w_terminal * bicycle_state_cost(x, cp);
    }
    case ORACLE_MODEL_QUADROTOR:
      return quad_state_cost(x, (const QuadrotorCostParams*)cost_params, 1);
    case ORACLE_MODEL_GUST:
      return 10.0 * (x[0] * x[0] + x[1] * x[1]);
    case ORACLE_MODEL_WEZ: { /* wez_environment.metal:222-240 */
      const WezCostParams* cp = (const WezCostParams*)cost_params;
      const double gx = x[0] - cp->x_goal, gy = x[1] - cp->y_goal;
      return cp->pos_weight * (gx * gx + gy * gy) * 10.0;
    }
    default: return 0.0;
  }
}

static inline double clampd(double v, double lo, double hi) {
  /* Metal clamp(x, lo, hi) = min(max(x, lo), hi) */
  const double a = v > lo ? v : lo;
  return a < hi ? a : hi;
}

/* Control-cost extension: lambda * u_nom_t^T Sigma^-1 eps_t. */
static double control_cost_term(const oracle_problem* p, const double* un, const double* e) {
  const uint32_t m = p->control_dim;
  double acc = 0.0;
  if (p->cov_full) {
    for (uint32_t i = 0; i < m; ++i)
      for (uint32_t j = 0; j < m; ++j) acc += un[i] * p->sigma_inv[i * m + j] * e[j];
  } else {
    for (uint32_t i = 0; i < m; ++i) acc += un[i] * p->sigma_inv[i] * e[i];
  }
  return p->lambda * acc;
}

/* ---- rollout (shaders/mppi_rollout.metal:36-96 / :103-170) ------------- */
void oracle_rollout(const oracle_problem* p, uint32_t step, uint32_t key,
                    const double* x0, const double* u_nom, const double* sigma,
                    const void* model_params, const void* cost_params, double* costs) {
  const uint32_t n = p->state_dim, m = p->control_dim, H = p->horizon;
  const uint32_t K = p->sample_count, P = (m + 1) / 2;
  double* eps = (double*)malloc(sizeof(double) * H * m);
  for (uint32_t k = 0; k < K; ++k) {
    double s[MAX_STATE];
    for (uint32_t d = 0; d < n && d < MAX_STATE; ++d) s[d] = x0[d];
    oracle_sample_noise(p, step, key, k, sigma, NULL, eps);
    double J = 0.0;
    for (uint32_t t = 0; t < H; ++t) {
      double u[MAX_CTRL];
      for (uint32_t d = 0; d < m; ++d)
        u[d] = clampd(u_nom[t * m + d] + eps[t * m + d], p->u_min[d], p->u_max[d]);
      if (p->control_cost) J += control_cost_term(p, u_nom + t * m, eps + t * m);
      /* dynamics counter: (step, k*H*P + t + 0x80000000)  (:89-90) */
      oracle_dynamics(p, s, u, model_params, step, k * H * P + t + 0x80000000u, key);
      J += oracle_stage_cost(p, s, u, model_params, cost_params); /* Q8 */
    }
    J += oracle_terminal_cost(p, s, model_params, cost_params);
    costs[k] = J;
  }
  free(eps);
}

void oracle_rollout_eps(const oracle_problem* p, const double* x0, const double* u_nom,
                        const void* model_params, const void* cost_params,
                        const double* eps_all, double* costs) {
  const uint32_t n = p->state_dim, m = p->control_dim, H = p->horizon, K = p->sample_count;
  for (uint32_t k = 0; k < K; ++k) {
    const double* eps = eps_all + (uint64_t)k * H * m;
    double s[MAX_STATE];
    for (uint32_t d = 0; d < n && d < MAX_STATE; ++d) s[d] = x0[d];
    double J = 0.0;
    for (uint32_t t = 0; t < H; ++t) {
      double u[MAX_CTRL];
      for (uint32_t d = 0; d < m; ++d)
        u[d] = clampd(u_nom[t * m + d] + eps[t * m + d], p->u_min[d], p->u_max[d]);
      if (p->control_cost) J += control_cost_term(p, u_nom + t * m, eps + t * m);
      oracle_dynamics(p, s, u, model_params, 0, 0, 0);
      J += oracle_stage_cost(p, s, u, model_params, cost_params);
    }
    J += oracle_terminal_cost(p, s, model_params, cost_params);
    costs[k] = J;
  }
}

void oracle_update_eps(const oracle_problem* p, const double* weights, const double* u_nom,
                       const double* eps_all, double* u_out) {
  const uint32_t m = p->control_dim, H = p->horizon, K = p->sample_count, L = H * m;
  for (uint32_t j = 0; j < L; ++j) {
    double acc = 0.0;
    for (uint32_t k = 0; k < K; ++k) acc += weights[k] * eps_all[(uint64_t)k * L + j];
    const uint32_t d = j % m;
    u_out[j] = clampd(u_nom[j] + acc, p->u_min[d], p->u_max[d]);
  }
}

/* ---- weights (shaders/mppi_reduce.metal:14-121) ------------------------- */
void oracle_weights(uint32_t K, double lambda, const double* costs, double* weights,
                    double diag[3]) {
  double mn = 1e38;
  for (uint32_t k = 0; k < K; ++k) mn = costs[k] < mn ? costs[k] : mn;
  double sw = 0.0, sc = 0.0;
  for (uint32_t k = 0; k < K; ++k) {
    const double w = exp(-(costs[k] - mn) / lambda);
    if (weights) weights[k] = w;
    sw += w;
    sc += costs[k];
  }
  double s2 = 0.0;
  for (uint32_t k = 0; k < K; ++k) {
    const double w = exp(-(costs[k] - mn) / lambda) / sw;
    if (weights) weights[k] = w;
    s2 += w * w;
  }
  diag[0] = mn;
  diag[1] = sc / (double)K;
  diag[2] = 1.0 / s2;
}

/* ---- update (shaders/mppi_reduce.metal:130-168) ------------------------- */
/* u_out = clamp(u_nom + sum_k w_k eps_k) with the UNCLAMPED noise (Q6). */
void oracle_update(const oracle_problem* p, uint32_t step, uint32_t key,
                   const double* weights, const double* u_nom, const double* sigma,
                   double* u_out) {
  const uint32_t m = p->control_dim, H = p->horizon, K = p->sample_count;
  const uint32_t L = H * m;
  double* acc = (double*)calloc(L, sizeof(double));
  double* eps = (double*)malloc(sizeof(double) * L);
  for (uint32_t k = 0; k < K; ++k) {
    oracle_sample_noise(p, step, key, k, sigma, NULL, eps);
    for (uint32_t j = 0; j < L; ++j) acc[j] += weights[k] * eps[j];
  }
  for (uint32_t j = 0; j < L; ++j) {
    const uint32_t d = j % m;
    u_out[j] = clampd(u_nom[j] + acc[j], p->u_min[d], p->u_max[d]);
  }
  free(acc);
  free(eps);
}

int oracle_step(const oracle_problem* p, uint32_t step, uint32_t key, const double* x0,
                const double* u_nom, double* u_out, double diag[3], double* costs_out,
                double* weights_out) {
  const uint32_t K = p->sample_count;
  double* costs = costs_out ? costs_out : (double*)malloc(sizeof(double) * K);
  double* w = weights_out ? weights_out : (double*)malloc(sizeof(double) * K);
  oracle_rollout(p, step, key, x0, u_nom, p->sigma, p->model_params, p->cost_params, costs);
  oracle_weights(K, p->lambda, costs, w, diag);
  oracle_update(p, step, key, w, u_nom, p->sigma, u_out);
  if (!costs_out) free(costs);
  if (!weights_out) free(w);
  return 0;
}

/* Shift left, hold last (src/mppi_driver.cpp:326-337; mppi_reduce.metal:221-230). */
static void shift_nominal(uint32_t H, uint32_t m, const double* u_opt, double* u_nom) {
  for (uint32_t t = 0; t < H; ++t) {
    const uint32_t src = (t + 1 < H) ? t + 1 : H - 1;
    for (uint32_t d = 0; d < m; ++d) u_nom[t * m + d] = u_opt[src * m + d];
  }
}

/* One agent's closed loop; prop_seed = 0 for simulate(), agent index for
 * simulate_batch() (mppi_reduce.metal:212-214, :467-468). */
static void closed_loop(const oracle_problem* p, uint32_t T, uint32_t start_step, uint32_t key,
                        uint32_t prop_seed, const double* sigma, const void* mp,
                        const void* cp, double* x, double* u_nom, uint32_t hist_stride,
                        uint32_t hist_off, double* states_out, double* controls_out,
                        double* costs_out) {
  const uint32_t n = p->state_dim, m = p->control_dim, H = p->horizon, K = p->sample_count;
  double* costs = (double*)malloc(sizeof(double) * K);
  double* w = (double*)malloc(sizeof(double) * K);
  double* u_out = (double*)malloc(sizeof(double) * H * m);
  for (uint32_t s = 0; s < T; ++s) {
    const uint32_t idx = start_step + s;
    double diag[3];
    oracle_rollout(p, idx, key, x, u_nom, sigma, mp, cp, costs);
    oracle_weights(K, p->lambda, costs, w, diag);
    oracle_update(p, idx, key, w, u_nom, sigma, u_out);
    /* propagate & shift (mppi_reduce.metal:175-231) */
    const uint64_t row = (uint64_t)s * hist_stride + hist_off;
    if (states_out)
      for (uint32_t d = 0; d < n; ++d) states_out[row * n + d] = x[d];
    if (controls_out)
      for (uint32_t d = 0; d < m; ++d) controls_out[row * m + d] = u_out[d];
    if (costs_out) costs_out[row] = diag[0];
    oracle_dynamics(p, x, u_out, mp, idx, 0x80000000u, prop_seed);
    shift_nominal(H, m, u_out, u_nom);
  }
  free(costs);
  free(w);
  free(u_out);
}

int oracle_simulate(const oracle_problem* p, uint32_t T, uint32_t start_step, uint32_t key,
                    const double* x0, const double* u_nom0, double* states_out,
                    double* controls_out, double* costs_out, double* x_final,
                    double* u_nom_final) {
  const uint32_t n = p->state_dim, L = p->horizon * p->control_dim;
  double x[MAX_STATE];
  double* u_nom = (double*)malloc(sizeof(double) * L);
  memcpy(x, x0, sizeof(double) * n);
  memcpy(u_nom, u_nom0, sizeof(double) * L);
  closed_loop(p, T, start_step, key, 0u, p->sigma, p->model_params, p->cost_params, x, u_nom,
              1, 0, states_out, controls_out, costs_out);
  if (x_final) memcpy(x_final, x, sizeof(double) * n);
  if (u_nom_final) memcpy(u_nom_final, u_nom, sizeof(double) * L);
  free(u_nom);
  return 0;
}

int oracle_simulate_batch(const oracle_problem* p, uint32_t N, uint32_t T, uint32_t start_step,
                          uint32_t seed, const oracle_agent_inputs* agents,
                          const double* x0_packed, const double* u_nom0_packed,
                          double* states_out, double* controls_out, double* costs_out,
                          double* terminal_out) {
  const uint32_t n = p->state_dim, m = p->control_dim, L = p->horizon * m;
  const uint32_t sig_len = p->cov_full ? m * m : m;
  double* u_nom = (double*)malloc(sizeof(double) * L);
  for (uint32_t a = 0; a < N; ++a) {
    double x[MAX_STATE];
    memcpy(x, x0_packed + (uint64_t)a * n, sizeof(double) * n);
    if (u_nom0_packed)
      memcpy(u_nom, u_nom0_packed + (uint64_t)a * L, sizeof(double) * L);
    else
      memset(u_nom, 0, sizeof(double) * L);
    const void* mp = p->model_params;
    const void* cp = p->cost_params;
    const double* sg = p->sigma;
    if (agents) {
      if (agents->model_params)
        mp = (const char*)agents->model_params + agents->model_stride * a;
      if (agents->cost_params)
        cp = (const char*)agents->cost_params + agents->cost_stride * a;
      if (agents->sigma) sg = agents->sigma + (uint64_t)a * sig_len;
    }
    closed_loop(p, T, start_step, seed + a, a, sg, mp, cp, x, u_nom, N, a, states_out,
                controls_out, costs_out);
    if (terminal_out) memcpy(terminal_out + (uint64_t)a * n, x, sizeof(double) * n);
  }
  free(u_nom);
  return 0;
}
