// driver_c.cpp — C ABI over mppi_metal::MPPIDriver (include/mppi_b200/mppi_driver_c.h).
#include "../../include/mppi_b200/mppi_driver_c.h"

#include <cstring>
#include <new>
#include <string>

#include "mppi_metal/mppi_driver.hpp"

using namespace mppi_metal;

struct mppi_driver {
  MPPIDriver driver;
  explicit mppi_driver(const DriverConfig& c, const DriverOptions& o) : driver(c, o) {}
};

namespace {

// Forwards a C++ error string into the caller's buffer (err may be NULL,
// exactly as the C++ API's std::string* error may be nullptr).
struct ErrSink {
  char* err;
  size_t len;
  std::string msg;
  std::string* ptr() { return err ? &msg : nullptr; }
  int done(bool ok) {
    if (!ok && err && len) {
      const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
      memcpy(err, msg.data(), n);
      err[n] = '\0';
    }
    return ok ? 1 : 0;
  }
};

}  // namespace

extern "C" {

mppi_driver* mppi_driver_create(const mppi_driver_config* c) {
  if (!c) return nullptr;
  DriverConfig cfg;
  cfg.state_dim = c->state_dim;
  cfg.control_dim = c->control_dim;
  cfg.horizon = c->horizon;
  cfg.sample_count = c->sample_count;
  cfg.lambda = c->lambda;
  cfg.noise.covariance_form = c->covariance_form == 1 ? ControlNoiseConfig::CovarianceForm::kFull
                                                      : ControlNoiseConfig::CovarianceForm::kDiagonal;
  cfg.noise.sigma = c->sigma;
  cfg.noise.sigma_inv = c->sigma_inv;
  cfg.noise.control_dim = c->noise_control_dim;
  cfg.bounds.u_min = c->u_min;
  cfg.bounds.u_max = c->u_max;
  cfg.bounds.control_dim = c->bounds_control_dim;
  cfg.numeric_mode = c->numeric_mode == 1   ? DriverConfig::NumericMode::kFp16
                     : c->numeric_mode == 2 ? DriverConfig::NumericMode::kMixed
                                            : DriverConfig::NumericMode::kFp32;
  DriverOptions opts;
  opts.control_cost = c->control_cost != 0;
  opts.proposal = c->proposal;
  opts.proposal_samples = c->proposal_samples;
  if (c->proposal_features && *c->proposal_features) opts.proposal_features = c->proposal_features;
  return new (std::nothrow) mppi_driver(cfg, opts);
}

void mppi_driver_destroy(mppi_driver* d) { delete d; }

int mppi_driver_initialize(mppi_driver* d, const mppi_driver_plugin* p, char* err,
                           size_t err_len) {
  ErrSink e{err, err_len, {}};
  if (!d || !p) {
    e.msg = "null argument.";
    return e.done(false);
  }
  ModelPluginSpec spec;
  spec.user_metallib_path = p->source_path ? p->source_path : "";
  const std::string dyn = p->dynamics ? p->dynamics : "mppi_dynamics";
  const std::string stage = p->stage_cost ? p->stage_cost : "";
  const std::string term = p->terminal_cost ? p->terminal_cost : "";
  spec.callables.dynamics = dyn;
  spec.callables.stage_cost = stage;
  spec.callables.terminal_cost = term;
  spec.param_layout.model_params_size = p->model_params_size;
  spec.param_layout.model_params_alignment = p->model_params_alignment ? p->model_params_alignment : 1;
  spec.param_layout.cost_params_size = p->cost_params_size;
  spec.param_layout.cost_params_alignment = p->cost_params_alignment ? p->cost_params_alignment : 1;
  spec.param_layout.schema_hash = p->schema_hash ? p->schema_hash : "";
  spec.rng.seed = p->seed;
  return e.done(d->driver.initialize(spec, e.ptr()));
}

int mppi_driver_set_problem_params(mppi_driver* d, const void* mp, size_t mpb, const void* cp,
                                   size_t cpb, char* err, size_t err_len) {
  ErrSink e{err, err_len, {}};
  ProblemParams pp;
  pp.model_params = {mp, mpb};
  pp.cost_params = {cp, cpb};
  return e.done(d->driver.set_problem_params(pp, e.ptr()));
}

int mppi_driver_step(mppi_driver* d, const float* x0, uint32_t x0_dim, const float* u_ovr,
                     uint32_t oh, uint32_t om, const void* mo, size_t mob, const void* co,
                     size_t cob, float* u_out, uint32_t out_h, uint32_t out_m, float* diag4,
                     char* err, size_t err_len) {
  ErrSink e{err, err_len, {}};
  StepInputs in;
  in.x0 = {x0, x0_dim};
  in.u_nominal_override = {u_ovr, oh, om};
  in.model_params_override = {mo, mob};
  in.cost_params_override = {co, cob};
  MutableControlSequenceView out{u_out, out_h, out_m};
  StepDiagnostics diag;
  const bool ok = d->driver.step(in, out, diag4 ? &diag : nullptr, e.ptr());
  if (ok && diag4) {
    diag4[0] = diag.best_cost;
    diag4[1] = diag.mean_cost;
    diag4[2] = diag.effective_sample_size;
    diag4[3] = diag.converged ? 1.0f : 0.0f;
  }
  return e.done(ok);
}

int mppi_driver_reset(mppi_driver* d, char* err, size_t err_len) {
  ErrSink e{err, err_len, {}};
  return e.done(d->driver.reset(e.ptr()));
}

int mppi_driver_reset_nominal(mppi_driver* d, const float* u, uint32_t h, uint32_t m, char* err,
                              size_t err_len) {
  ErrSink e{err, err_len, {}};
  return e.done(d->driver.reset(ControlSequenceView{u, h, m}, e.ptr()));
}

int mppi_driver_simulate(mppi_driver* d, uint32_t T, const float* x0, uint32_t x0_dim,
                         const float* u_ovr, uint32_t oh, uint32_t om, const void* mo,
                         size_t mob, const void* co, size_t cob, float* states, float* controls,
                         float* costs, uint32_t res_steps, char* err, size_t err_len) {
  ErrSink e{err, err_len, {}};
  StepInputs in;
  in.x0 = {x0, x0_dim};
  in.u_nominal_override = {u_ovr, oh, om};
  in.model_params_override = {mo, mob};
  in.cost_params_override = {co, cob};
  SimulationResults r;
  r.states_out = states;
  r.controls_out = controls;
  r.costs_out = costs;
  r.num_steps = res_steps;
  return e.done(d->driver.simulate(T, in, r, e.ptr()));
}

int mppi_driver_simulate_batch(mppi_driver* d, uint32_t N, uint32_t T, const float* x0,
                               float* states, float* controls, float* costs, float* terminal,
                               uint32_t res_agents, uint32_t res_steps, char* err,
                               size_t err_len) {
  ErrSink e{err, err_len, {}};
  BatchSimulationResults r;
  r.states_out = states;
  r.controls_out = controls;
  r.costs_out = costs;
  r.terminal_states_out = terminal;
  r.num_agents = res_agents;
  r.num_steps = res_steps;
  return e.done(d->driver.simulate_batch(N, T, x0, r, e.ptr()));
}

int mppi_driver_simulate_batch_agents(mppi_driver* d, uint32_t N, uint32_t T, const float* x0,
                                      const void* mp, size_t mps, const void* cp, size_t cps,
                                      const float* sigma, const uint32_t* sample_counts,
                                      const uint32_t* horizons, float* states, float* controls,
                                      float* costs, float* terminal, uint32_t res_agents,
                                      uint32_t res_steps, char* err, size_t err_len) {
  ErrSink e{err, err_len, {}};
  BatchAgentParams ap;
  ap.model_params = mp;
  ap.model_params_stride = mps;
  ap.cost_params = cp;
  ap.cost_params_stride = cps;
  ap.sigma = sigma;
  ap.sample_counts = sample_counts;
  ap.horizons = horizons;
  BatchSimulationResults r;
  r.states_out = states;
  r.controls_out = controls;
  r.costs_out = costs;
  r.terminal_states_out = terminal;
  r.num_agents = res_agents;
  r.num_steps = res_steps;
  return e.done(d->driver.simulate_batch(N, T, x0, ap, r, e.ptr()));
}

}  // extern "C"
