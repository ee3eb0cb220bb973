/*
 * mppi_oracle — FP64 CPU restatement of the reference MPPI hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker.
 * The product (libmppi_b200.so) never links or calls it.
 *
 * What it restates (reference = MarshallVielmetti/mppi_metal):
 *   - Philox-2x32-10 words, bit-exact            shaders/philox.h:19-36
 *   - uint -> (0,1) map and Box-Muller            shaders/philox.h:39-50
 *   - rollout (noise, clamp, dynamics, costs)     shaders/mppi_rollout.metal:36-170
 *   - softmax weights + diagnostics               shaders/mppi_reduce.metal:14-121
 *   - weighted-noise update                       shaders/mppi_reduce.metal:130-168
 *   - propagate & shift                           shaders/mppi_reduce.metal:175-231,413-488
 *   - driver warm start / step index / batch      src/mppi_driver.cpp:235-341,423-491
 * plus the documented extensions of this project (full-covariance Cholesky
 * shaping, the lambda * u^T Sigma^-1 eps control cost, per-agent parameter
 * blobs and sigma), which have no reference counterpart.
 *
 * Arithmetic: Philox words in exact uint32; the uniform map is evaluated in
 * float exactly as the reference defines it ((float(x) + 0.5f) * 2^-32, two
 * correctly rounded float operations, so it is bit-exact); everything after
 * it (log, sqrt, sin, cos, dynamics, costs, weights, sums) runs in double.
 *
 * Pinning: the Philox words and the whole FP32 pipeline are checked against
 * the reference's own shader sources compiled for the CPU (oracle/_ref, see
 * oracle/Makefile) through committed golden vectors in tests/golden/.
 */
#ifndef MPPI_ORACLE_H
#define MPPI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Model restatements (one per plugin in mppi_metal_b200/plugins). */
enum {
  ORACLE_MODEL_DOUBLE_INTEGRATOR = 0,
  ORACLE_MODEL_NONHOLONOMIC = 1,
  ORACLE_MODEL_UNICYCLE_OBSTACLES = 2,
  ORACLE_MODEL_BICYCLE_LANE = 3,
  ORACLE_MODEL_QUADROTOR = 4,
  ORACLE_MODEL_GUST = 5,
  ORACLE_MODEL_WEZ = 6,
};

typedef struct {
  uint32_t state_dim;
  uint32_t control_dim;
  uint32_t horizon;
  uint32_t sample_count;
  double lambda;
  int32_t cov_full;     /* 0: sigma = per-dim std-dev; 1: sigma = m*m covariance */
  int32_t control_cost; /* 1: add lambda * u_nom^T Sigma^-1 eps per time step */
  int32_t model;        /* ORACLE_MODEL_* */
  int32_t use_stage;    /* 0: library default stage cost (returns 0) */
  int32_t use_terminal; /* 0: library default terminal cost (returns 0) */
  int32_t noise_half;   /* 1: shaped noise rounded to IEEE binary16 (kFp16 / kMixed) */
  const double* sigma;     /* m (diag) or m*m (full, row-major covariance) */
  const double* sigma_inv; /* m or m*m; read only when control_cost != 0 */
  const double* u_min;     /* m */
  const double* u_max;     /* m */
  const void* model_params; /* float blob (plugins/model_params.h) */
  const void* cost_params;  /* float blob */
} oracle_problem;

/* Per-agent inputs for the batch paths.  Null pointers / zero strides mean
 * "shared by all agents" (the reference's batch semantics). */
typedef struct {
  const void* model_params;   /* base of the packed blobs */
  uint64_t model_stride;      /* bytes between agents (0 = shared) */
  const void* cost_params;
  uint64_t cost_stride;
  const double* sigma;        /* [N][m] or [N][m*m]; null = problem sigma */
} oracle_agent_inputs;

/* ---- RNG ---------------------------------------------------------------- */
void oracle_philox2x32_10(uint32_t c0, uint32_t c1, uint32_t key, uint32_t out[2]);
void oracle_philox_many(uint64_t n, const uint32_t* c0, const uint32_t* c1,
                        const uint32_t* key, uint32_t* out /* [n][2] */);
float oracle_uint_to_01(uint32_t x);
void oracle_box_muller(uint32_t w0, uint32_t w1, double out[2]);

/* Standard normals n[t][d] (H*m, before shaping) and shaped noise
 * eps[t][d] for sample k; either output may be null. */
void oracle_sample_noise(const oracle_problem* p, uint32_t step, uint32_t key,
                         uint32_t k, const double* sigma, double* normals,
                         double* eps);

/* ---- passes ------------------------------------------------------------- */
void oracle_rollout(const oracle_problem* p, uint32_t step, uint32_t key,
                    const double* x0, const double* u_nom, const double* sigma,
                    const void* model_params, const void* cost_params,
                    double* costs /* K */);
void oracle_weights(uint32_t K, double lambda, const double* costs,
                    double* weights /* K, may be null */, double diag[3]);
void oracle_update(const oracle_problem* p, uint32_t step, uint32_t key,
                   const double* weights, const double* u_nom,
                   const double* sigma, double* u_out /* H*m */);
void oracle_dynamics(const oracle_problem* p, double* x, const double* u,
                     const void* model_params, uint32_t ctr0, uint32_t ctr1,
                     uint32_t key);
double oracle_stage_cost(const oracle_problem* p, const double* x,
                         const double* u, const void* model_params,
                         const void* cost_params);
double oracle_terminal_cost(const oracle_problem* p, const double* x,
                            const void* model_params, const void* cost_params);

/* The rollout and the update on a given noise array eps[K][H][m] (for
 * checking a device pass against the oracle on the device's own noise). */
void oracle_rollout_eps(const oracle_problem* p, const double* x0, const double* u_nom,
                        const void* model_params, const void* cost_params,
                        const double* eps_all, double* costs);
void oracle_update_eps(const oracle_problem* p, const double* weights, const double* u_nom,
                       const double* eps_all, double* u_out);

/* One control step for one agent: rollout -> weights -> update. */
int oracle_step(const oracle_problem* p, uint32_t step, uint32_t key,
                const double* x0, const double* u_nom, double* u_out,
                double diag[3], double* costs_out, double* weights_out);

/* Closed loop for one agent (MPPIDriver::simulate).  History is indexed by
 * the local step (0..T-1).  Outputs may be null. */
int oracle_simulate(const oracle_problem* p, uint32_t T, uint32_t start_step,
                    uint32_t key, const double* x0, const double* u_nom0,
                    double* states_out, double* controls_out,
                    double* costs_out, double* x_final, double* u_nom_final);

/* Closed loop for N agents (MPPIDriver::simulate_batch): agent a uses key
 * seed + a and propagation seed a; all agents start from u_nom0 (the
 * reference passes zeros).  Histories are step-major [T][N][dim]. */
int oracle_simulate_batch(const oracle_problem* p, uint32_t N, uint32_t T,
                          uint32_t start_step, uint32_t seed,
                          const oracle_agent_inputs* agents,
                          const double* x0_packed, const double* u_nom0_packed,
                          double* states_out, double* controls_out,
                          double* costs_out, double* terminal_out);

/* Lower-triangular Cholesky factor of an m*m SPD matrix (row-major). */
int oracle_cholesky(uint32_t m, const double* a, double* l);

#ifdef __cplusplus
}
#endif

#endif /* MPPI_ORACLE_H */
