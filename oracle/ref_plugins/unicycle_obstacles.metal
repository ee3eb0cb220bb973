// unicycle_obstacles.metal — the unicycle-among-moving-obstacles model written
// against the reference's MSL plugin contract (shaders/mppi_core.h:11-26), so
// the reference's own kernels can run the benchmark workload.  Compiles with
// the Metal compiler, and as C++ through oracle/ref_shim for the CPU harness.
// Same model as mppi_metal_b200/plugins/unicycle_obstacles.cu and the oracle.
#include <metal_stdlib>
#include "mppi_core.h"
#include "model_params.h"

using namespace metal;

[[visible]]
void mppi_dynamics(thread uint8_t* state_raw, thread const float* control,
                   device const uint8_t* model_params_raw, uint2 rng_counter, uint rng_seed) {
    device const UnicycleModelParams* mp = (device const UnicycleModelParams*)model_params_raw;
    thread float* s = (thread float*)state_raw;
    float dt = mp->dt;
    float th = s[2];
    s[0] += control[0] * cos(th) * dt;
    s[1] += control[0] * sin(th) * dt;
    s[2] += control[1] * dt;
    s[3] += dt;
}

static float unicycle_goal_cost(thread const float* s, device const UnicycleCostParams* cp) {
    float dx = s[0] - cp->goal_x;
    float dy = s[1] - cp->goal_y;
    return cp->w_goal * (dx * dx + dy * dy);
}

[[visible]]
float mppi_stage_cost(thread const uint8_t* state_raw, thread const float* control,
                      device const uint8_t* model_params_raw, device const uint8_t* cost_params_raw) {
    device const UnicycleCostParams* cp = (device const UnicycleCostParams*)cost_params_raw;
    thread const float* s = (thread const float*)state_raw;
    float pen = 0.0f;
    float t = s[3];
    for (uint i = 0; i < cp->num_obs && i < MPPI_UNICYCLE_MAX_OBS; ++i) {
        float cx = cp->obs_cx[i] + cp->obs_vx[i] * t;
        float cy = cp->obs_cy[i] + cp->obs_vy[i] * t;
        float ex = s[0] - cx;
        float ey = s[1] - cy;
        float v = cp->obs_r[i] - sqrt(ex * ex + ey * ey);
        pen += max(v, 0.0f);
    }
    return unicycle_goal_cost(s, cp) + cp->w_obs * pen;
}

[[visible]]
float mppi_terminal_cost(thread const uint8_t* state_raw, device const uint8_t* model_params_raw,
                         device const uint8_t* cost_params_raw) {
    device const UnicycleCostParams* cp = (device const UnicycleCostParams*)cost_params_raw;
    thread const float* s = (thread const float*)state_raw;
    return cp->w_terminal * unicycle_goal_cost(s, cp);
}
