// ref_harness.cpp — runs the REFERENCE's own kernels on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into oracle/_ref/ from
// the reference's shader sources (shaders/mppi_rollout.metal,
// shaders/mppi_reduce.metal, shaders/philox.h, shaders/mppi_core.h) compiled
// as C++ through oracle/ref_shim/metal_stdlib, together with one model plugin
// (a reference plugin such as shaders/test_user_dynamics.metal, or an MSL
// plugin from oracle/ref_plugins/).  Nothing of the reference is copied here:
// this file only declares the kernels' entry points and replays the
// dispatch sequences of src/metal_backend.mm:
//   dispatch_rollout           metal_backend.mm:604-741  (rollout, weights, reduce)
//   dispatch_simulation        metal_backend.mm:747-929  (+ propagate & shift, T times)
//   dispatch_batch_simulation  metal_backend.mm:935-1124 (batch kernels, T times)
// with a CPU "grid": every kernel invocation is one call per thread index.
// Work is split over host threads by sample (rollout) and by output element
// (reduce); the weights kernel runs as a one-thread threadgroup, a valid
// schedule of it (its loops stride by the threadgroup size).
//
// Per-agent parameter blobs and sigma (a project extension the reference's
// batch API lacks) are emulated by handing the batch kernels a different
// params / sigma pointer for each agent row of the grid.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include <metal_stdlib>

#include "mppi_core.h"

// The shim's address-space macros are only needed for the reference headers.
#undef device
#undef thread
#undef threadgroup
#undef constant

using metal::visible_function_table;
using DynTable = visible_function_table<MppiDynamicsFn>;
using StageTable = visible_function_table<MppiStageCostFn>;
using TermTable = visible_function_table<MppiTerminalCostFn>;

// ---- entry points of the reference kernels (defined in the .metal TUs) ----
void mppi_rollout(const float*, const float*, const uint8_t*, const uint8_t*, float*,
                  const uint&, const uint&, const uint&, const uint&, const float*,
                  const float*, DynTable, StageTable, TermTable, const float*, const uint&,
                  const uint&, uint);
void mppi_rollout_batch(const float*, const float*, const uint8_t*, const uint8_t*, float*,
                        const uint&, const uint&, const uint&, const uint&, const float*,
                        const float*, DynTable, StageTable, TermTable, const float*,
                        const uint&, const uint&, const uint&, uint2);
float mppi_default_stage_cost(const uint8_t*, const float*, const uint8_t*, const uint8_t*);
float mppi_default_terminal_cost(const uint8_t*, const uint8_t*, const uint8_t*);
void mppi_compute_weights(const float*, float*, float*, const uint&, const float&, uint, uint,
                          uint, uint);
void mppi_compute_weights_batch(const float*, float*, float*, const uint&, const float&,
                                const uint&, uint, uint, uint, uint, uint);
void mppi_reduce(const float*, const float*, float*, const float*, const float*, const float*,
                 const uint&, const uint&, const uint&, const uint&, const uint&, uint);
void mppi_reduce_batch(const float*, const float*, float*, const float*, const float*,
                       const float*, const uint&, const uint&, const uint&, const uint&,
                       const uint&, const uint&, uint2);
void mppi_propagate_and_shift(float*, float*, const float*, float*, float*, float*,
                              const float*, const uint8_t*, const uint&, const uint&,
                              const uint&, const uint&, DynTable, uint);
void mppi_propagate_and_shift_batch(float*, float*, const float*, float*, float*, float*,
                                    const float*, const uint8_t*, const uint&, const uint&,
                                    const uint&, const uint&, DynTable, const uint&,
                                    const uint&, float*, uint2);

// ---- the plugin's callables (oracle/ref_plugin_adapter.cpp) --------------
extern "C" void* ref_plugin_dynamics();
extern "C" void* ref_plugin_stage_cost();
extern "C" void* ref_plugin_terminal_cost();

extern "C" {

struct ref_config {
  uint32_t state_dim;
  uint32_t control_dim;
  uint32_t horizon;
  uint32_t sample_count;
  float lambda;
  uint32_t seed;       // ModelPluginSpec::rng.seed truncated to 32 bits (metal_backend.mm:565)
  int32_t use_stage;   // 0: the library's default stage cost
  int32_t use_terminal;
  int32_t nthreads;
  int32_t pad;
};

}  // extern "C"

namespace {

struct Tables {
  DynTable dyn;
  StageTable stage;
  TermTable term;
};

Tables make_tables(const ref_config* c) {
  Tables t;
  t.dyn.fn = reinterpret_cast<MppiDynamicsFn*>(ref_plugin_dynamics());
  t.stage.fn = c->use_stage ? reinterpret_cast<MppiStageCostFn*>(ref_plugin_stage_cost())
                            : &mppi_default_stage_cost;
  t.term.fn = c->use_terminal ? reinterpret_cast<MppiTerminalCostFn*>(ref_plugin_terminal_cost())
                              : &mppi_default_terminal_cost;
  return t;
}

template <class F>
void parallel_for(uint32_t n, int nthreads, F&& f) {
  const uint32_t nt = std::max(1, std::min<int>(nthreads, (int)std::max<uint32_t>(n, 1)));
  if (nt == 1) {
    for (uint32_t i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (uint32_t w = 0; w < nt; ++w) {
    th.emplace_back([&, w] {
      const uint64_t lo = (uint64_t)n * w / nt, hi = (uint64_t)n * (w + 1) / nt;
      for (uint64_t i = lo; i < hi; ++i) f((uint32_t)i);
    });
  }
  for (auto& t : th) t.join();
}

const uint8_t kZeroByte[16] = {0};

const uint8_t* param_or_zero(const void* p) {
  // metal_backend.mm:595-600: an unbound params slot gets a 1-byte zero buffer.
  return p ? static_cast<const uint8_t*>(p) : kZeroByte;
}

}  // namespace

extern "C" {

// dispatch_rollout (metal_backend.mm:604-741): rollout -> weights -> reduce.
int ref_step(const ref_config* c, uint32_t step_index, const float* x0, const float* u_nom,
             const float* sigma, const float* u_min, const float* u_max, const void* mp,
             const void* cp, float* u_out, float* diag3, float* costs_out, float* weights_out) {
  const uint S = c->sample_count, H = c->horizon, sdim = c->state_dim, cdim = c->control_dim;
  const uint seed = c->seed, step = step_index, L = H * cdim;
  const float lambda = c->lambda;
  Tables tb = make_tables(c);
  std::vector<float> costs(S), weights(S);
  float diag[3];
  const uint8_t* mpb = param_or_zero(mp);
  const uint8_t* cpb = param_or_zero(cp);
  parallel_for(S, c->nthreads, [&](uint32_t gid) {
    mppi_rollout(x0, u_nom, mpb, cpb, costs.data(), sdim, cdim, H, S, u_min, u_max, tb.dyn,
                 tb.stage, tb.term, sigma, seed, step, gid);
  });
  mppi_compute_weights(costs.data(), weights.data(), diag, S, lambda, 0, 1, 0, 0);
  parallel_for(L, c->nthreads, [&](uint32_t gid) {
    mppi_reduce(weights.data(), u_nom, u_out, sigma, u_min, u_max, S, H, cdim, seed, step, gid);
  });
  if (diag3) std::memcpy(diag3, diag, sizeof(diag));
  if (costs_out) std::memcpy(costs_out, costs.data(), sizeof(float) * S);
  if (weights_out) std::memcpy(weights_out, weights.data(), sizeof(float) * S);
  return 0;
}

// dispatch_simulation (metal_backend.mm:747-929).  The reference indexes the
// history by the absolute step index; the harness sizes its history for
// start + T rows and returns the last T so it never writes out of bounds.
int ref_simulate(const ref_config* c, uint32_t T, uint32_t start_step, const float* x0,
                 const float* u_nom0, const float* sigma, const float* u_min,
                 const float* u_max, const void* mp, const void* cp, float* states_out,
                 float* controls_out, float* costs_out) {
  const uint S = c->sample_count, H = c->horizon, sdim = c->state_dim, cdim = c->control_dim;
  const uint seed = c->seed, L = H * cdim;
  const float lambda = c->lambda;
  Tables tb = make_tables(c);
  const uint8_t* mpb = param_or_zero(mp);
  const uint8_t* cpb = param_or_zero(cp);
  std::vector<float> x(x0, x0 + sdim), u_nom(u_nom0, u_nom0 + L), u_out(L), costs(S),
      weights(S), diag(3);
  const uint64_t rows = (uint64_t)start_step + T;
  std::vector<float> hs(rows * sdim), hc(rows * cdim), hk(rows);
  for (uint32_t s = 0; s < T; ++s) {
    const uint step = start_step + s;
    parallel_for(S, c->nthreads, [&](uint32_t gid) {
      mppi_rollout(x.data(), u_nom.data(), mpb, cpb, costs.data(), sdim, cdim, H, S, u_min,
                   u_max, tb.dyn, tb.stage, tb.term, sigma, seed, step, gid);
    });
    mppi_compute_weights(costs.data(), weights.data(), diag.data(), S, lambda, 0, 1, 0, 0);
    parallel_for(L, c->nthreads, [&](uint32_t gid) {
      mppi_reduce(weights.data(), u_nom.data(), u_out.data(), sigma, u_min, u_max, S, H, cdim,
                  seed, step, gid);
    });
    for (uint gid = 0; gid < L; ++gid)
      mppi_propagate_and_shift(x.data(), u_nom.data(), u_out.data(), hs.data(), hc.data(),
                               hk.data(), diag.data(), mpb, sdim, cdim, H, step, tb.dyn, gid);
  }
  if (states_out) std::memcpy(states_out, hs.data() + (uint64_t)start_step * sdim, sizeof(float) * T * sdim);
  if (controls_out) std::memcpy(controls_out, hc.data() + (uint64_t)start_step * cdim, sizeof(float) * T * cdim);
  if (costs_out) std::memcpy(costs_out, hk.data() + start_step, sizeof(float) * T);
  return 0;
}

// dispatch_batch_simulation (metal_backend.mm:935-1124) with optional
// per-agent params / sigma (strides in bytes / floats; 0 = shared).
int ref_simulate_batch(const ref_config* c, uint32_t N, uint32_t T, uint32_t start_step,
                       const float* x0_packed, const float* u_nom0_packed, const float* sigma,
                       uint64_t sigma_stride, const float* u_min, const float* u_max,
                       const void* mp, uint64_t mp_stride, const void* cp, uint64_t cp_stride,
                       float* states_out, float* controls_out, float* costs_out,
                       float* terminal_out) {
  const uint S = c->sample_count, H = c->horizon, sdim = c->state_dim, cdim = c->control_dim;
  const uint seed = c->seed, L = H * cdim, NA = N, TT = T;
  const float lambda = c->lambda;
  Tables tb = make_tables(c);
  std::vector<float> x(x0_packed, x0_packed + (uint64_t)N * sdim);
  std::vector<float> u_nom((uint64_t)N * L, 0.0f), u_out((uint64_t)N * L);
  if (u_nom0_packed) std::memcpy(u_nom.data(), u_nom0_packed, sizeof(float) * N * L);
  std::vector<float> costs((uint64_t)N * S), weights((uint64_t)N * S), diag((uint64_t)N * 3);
  const uint64_t rows = (uint64_t)start_step + T;
  std::vector<float> hs(rows * N * sdim), hc(rows * N * cdim), hk(rows * N), term((uint64_t)N * sdim);
  auto agent_mp = [&](uint32_t a) {
    return param_or_zero(mp ? static_cast<const uint8_t*>(mp) + mp_stride * a : nullptr);
  };
  auto agent_cp = [&](uint32_t a) {
    return param_or_zero(cp ? static_cast<const uint8_t*>(cp) + cp_stride * a : nullptr);
  };
  auto agent_sigma = [&](uint32_t a) { return sigma + sigma_stride * a; };
  for (uint32_t s = 0; s < T; ++s) {
    const uint step = start_step + s;
    parallel_for(N * S, c->nthreads, [&](uint32_t i) {
      const uint32_t a = i / S, k = i % S;
      mppi_rollout_batch(x.data(), u_nom.data(), agent_mp(a), agent_cp(a), costs.data(), sdim,
                         cdim, H, S, u_min, u_max, tb.dyn, tb.stage, tb.term, agent_sigma(a),
                         seed, step, NA, uint2(k, a));
    });
    parallel_for(N, c->nthreads, [&](uint32_t a) {
      mppi_compute_weights_batch(costs.data(), weights.data(), diag.data(), S, lambda, NA, 0, 1,
                                 0, 0, a);
    });
    parallel_for(N * L, c->nthreads, [&](uint32_t i) {
      const uint32_t a = i / L, j = i % L;
      mppi_reduce_batch(weights.data(), u_nom.data(), u_out.data(), agent_sigma(a), u_min,
                        u_max, S, H, cdim, seed, step, NA, uint2(j, a));
    });
    parallel_for(N, c->nthreads, [&](uint32_t a) {
      for (uint j = 0; j < L; ++j)
        mppi_propagate_and_shift_batch(x.data(), u_nom.data(), u_out.data(), hs.data(),
                                       hc.data(), hk.data(), diag.data(), agent_mp(a), sdim,
                                       cdim, H, step, tb.dyn, NA, TT, term.data(), uint2(j, a));
    });
  }
  if (states_out)
    std::memcpy(states_out, hs.data() + (uint64_t)start_step * N * sdim, sizeof(float) * T * N * sdim);
  if (controls_out)
    std::memcpy(controls_out, hc.data() + (uint64_t)start_step * N * cdim, sizeof(float) * T * N * cdim);
  if (costs_out) std::memcpy(costs_out, hk.data() + (uint64_t)start_step * N, sizeof(float) * T * N);
  if (terminal_out) std::memcpy(terminal_out, term.data(), sizeof(float) * N * sdim);
  return 0;
}

// Raw Philox-2x32-10 words and Box-Muller pairs from shaders/philox.h.
void ref_philox_words(uint64_t n, const uint32_t* c0, const uint32_t* c1, const uint32_t* key,
                      uint32_t* out);
void ref_box_muller(uint64_t n, const uint32_t* words, float* out);

}  // extern "C"
