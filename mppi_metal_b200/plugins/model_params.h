/*
 * Parameter-blob layouts of the model plugins shipped with mppi_metal_b200.
 *
 * One plain-C header shared by three consumers, so a blob built on the host
 * means the same thing everywhere:
 *   - the CUDA plugins in this directory (compiled by NVRTC into the rollout
 *     kernel; the blob reaches them as `const uint8_t* model_params/cost_params`),
 *   - the FP64 oracle (oracle/mppi_oracle.c), which restates each model,
 *   - the MSL plugins under oracle/ref_plugins (run through the reference's
 *     own kernels on the CPU for the timed reference baseline).
 * Python mirrors live in mppi_metal_b200/models.py (ctypes structures).
 *
 * Every field is a 4-byte float or uint32 so the layout is identical under
 * gcc, nvcc/NVRTC and the Metal compiler.
 */
#ifndef MPPI_B200_MODEL_PARAMS_H
#define MPPI_B200_MODEL_PARAMS_H

/* ------------------------------------------------------------------------ */
/* double_integrator: the reference's test model                             */
/* (shaders/test_user_dynamics.metal:8-43).  State [px, py, vx, vy],        */
/* control [ax, ay], dt fixed at 0.1, stage = terminal = px^2 + py^2.        */
/* No parameter blobs.                                                       */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* nonholonomic_vehicle: the reference example model                         */
/* (examples/nonholonomic_vehicle/nonholonomic_vehicle.metal:6-91).          */
/* State [x, y, theta, v], control [a, omega].  Field order kept so blobs    */
/* built for the reference example bind unchanged.                           */
/* ------------------------------------------------------------------------ */
typedef struct {
  float v_max;
  float dt;
} NonholonomicModelParams;

typedef struct {
  float x_goal;
  float y_goal;
  float goal_radius;
  float pos_weight;
  float heading_weight;
  float control_weight;
} NonholonomicCostParams;

/* ------------------------------------------------------------------------ */
/* unicycle_obstacles: kinematic unicycle among moving circular keep-out     */
/* regions.  State [x, y, theta, t] (t = model time, advanced by dt so that  */
/* obstacle positions c_i + v_i * t follow the closed loop), control         */
/* [v, omega].                                                               */
/*   dynamics : x += v cos(theta) dt; y += v sin(theta) dt;                  */
/*              theta += omega dt; t += dt                                   */
/*   stage    : w_goal * |p - g|^2 + w_obs * sum_i max(0, r_i - |p - c_i(t)|)*/
/*   terminal : w_terminal * w_goal * |p - g|^2                              */
/* ------------------------------------------------------------------------ */
#define MPPI_UNICYCLE_MAX_OBS 16

typedef struct {
  float dt;
  float pad0;
  float pad1;
  float pad2;
} UnicycleModelParams;

typedef struct {
  float goal_x;
  float goal_y;
  float w_goal;
  float w_obs;
  float w_terminal;
  unsigned int num_obs;
  float pad0;
  float pad1;
  /* structure-of-arrays so the cost loop reads 16-byte vectors */
  float obs_cx[MPPI_UNICYCLE_MAX_OBS];
  float obs_cy[MPPI_UNICYCLE_MAX_OBS];
  float obs_vx[MPPI_UNICYCLE_MAX_OBS];
  float obs_vy[MPPI_UNICYCLE_MAX_OBS];
  float obs_r[MPPI_UNICYCLE_MAX_OBS];
} UnicycleCostParams;

/* ------------------------------------------------------------------------ */
/* bicycle_lane: kinematic bicycle tracking a cubic-spline lane centreline.  */
/* State [x, y, theta, v, delta], control [accel, steer_rate].               */
/*   dynamics : x += v cos(theta) dt; y += v sin(theta) dt;                  */
/*              theta += v / wheelbase * tan(delta) dt; v += a dt;           */
/*              delta = clamp(delta + steer_rate dt, -delta_max, delta_max)  */
/*   centreline y_c(x): natural cubic spline over knots x_0 + i * knot_dx,   */
/*   segment i holds y = c0 + c1 s + c2 s^2 + c3 s^3 with s = x - x_i; x is  */
/*   clamped to the knot range.                                              */
/*   stage    : w_lat (y - y_c)^2 + w_head (theta - atan(y_c'))^2            */
/*              + w_speed (v - v_ref)^2                                      */
/*   terminal : w_terminal * (state part of stage)                           */
/* ------------------------------------------------------------------------ */
#define MPPI_BICYCLE_MAX_SEGMENTS 32

typedef struct {
  float dt;
  float wheelbase;
  float delta_max;
  float pad0;
} BicycleModelParams;

typedef struct {
  float x0;
  float knot_dx;
  unsigned int num_segments;
  float v_ref;
  float w_lat;
  float w_head;
  float w_speed;
  float w_terminal;
  float coef[MPPI_BICYCLE_MAX_SEGMENTS][4];
} BicycleCostParams;

/* ------------------------------------------------------------------------ */
/* quadrotor: 12-state rigid-body quadrotor with 4 rotor thrusts.            */
/* State [px,py,pz, vx,vy,vz, phi,theta,psi, p,q,r], control [f1..f4].       */
/*   thrust T = f1+f2+f3+f4 along body z; torques (plus layout, arm l,       */
/*   yaw coefficient k): tx = l (f2 - f4), ty = l (f3 - f1),                 */
/*   tz = k (f1 - f2 + f3 - f4); inertia diag(Jx, Jy, Jz).                   */
/*   v' = R(phi,theta,psi) [0,0,T/mass] - [0,0,g];  euler' = W(phi,theta) w;  */
/*   w' = J^-1 (tau - w x J w); explicit Euler with dt.                      */
/*   stage    : w_pos |p - wp|^2 + w_vel |v|^2 + w_att (phi^2 + theta^2)     */
/*              + w_rate |w|^2 + w_obs sum_i max(0, r_i - |p - c_i|)          */
/*   terminal : w_terminal * w_pos |p - wp|^2                                */
/* ------------------------------------------------------------------------ */
#define MPPI_QUAD_MAX_OBS 32

typedef struct {
  float dt;
  float mass;
  float gravity;
  float arm;
  float yaw_coef;
  float jx;
  float jy;
  float jz;
} QuadrotorModelParams;

typedef struct {
  float wp_x;
  float wp_y;
  float wp_z;
  float w_pos;
  float w_vel;
  float w_att;
  float w_rate;
  float w_obs;
  float w_terminal;
  unsigned int num_obs;
  float pad0;
  float pad1;
  float obs_cx[MPPI_QUAD_MAX_OBS];
  float obs_cy[MPPI_QUAD_MAX_OBS];
  float obs_cz[MPPI_QUAD_MAX_OBS];
  float obs_r[MPPI_QUAD_MAX_OBS];
} QuadrotorCostParams;

/* ------------------------------------------------------------------------ */
/* gust_integrator: stochastic dynamics (draws its own Philox randoms from  */
/* the callable's rng_counter / rng_seed, as the reference's WEZ example    */
/* does, examples/wez_environment_batch/wez_environment.metal:166-173).     */
/* State [px, py, vx, vy, gust], control [ax, ay].                          */
/*   n = box_muller(philox(rng_counter, rng_seed))                           */
/*   e = uint_to_01(philox((ctr.x, ctr.y + 0x1000), rng_seed).x)             */
/*   gust = 1 once e < p_event (sticky)                                      */
/*   v += (u + noise_std * n + gust * (gust_accel, 0)) dt;  p += v dt        */
/*   stage = px^2 + py^2 + 0.1 |v|^2;  terminal = 10 (px^2 + py^2)           */
/* ------------------------------------------------------------------------ */
typedef struct {
  float dt;
  float noise_std;
  float p_event;
  float gust_accel;
} GustModelParams;

/* ------------------------------------------------------------------------ */
/* wez_environment: the reference's stochastic example                       */
/* (examples/wez_environment_batch/wez_environment.metal:8-32,               */
/* examples/wez_environment_batch/main.cpp:11-37).  Field order kept so the  */
/* example's blobs bind unchanged.  State and formulas: wez_environment.cu.  */
/* ------------------------------------------------------------------------ */
typedef struct {
  float v_max;
  float dt;
  float adv_v_max;
  float adv_fire_prob_max;
  float adv_max_range;
  float adv_min_range;
  float adv_k_gain;
  float adv_capture_radius;
  int adv_max_steps;
  int num_adversaries;
} WezModelParams;

typedef struct {
  float x_goal;
  float y_goal;
  float goal_radius;
  float pos_weight;
  float heading_weight;
  float control_weight;
  float adv_collision_weight;
  float adv_dist_weight;
} WezCostParams;

#endif /* MPPI_B200_MODEL_PARAMS_H */
