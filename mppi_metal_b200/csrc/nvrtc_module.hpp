// nvrtc_module.hpp — per-driver kernel module: the library kernel template
// (csrc/device/*.cuh, embedded in this library) compiled together with the
// user's plugin source by NVRTC for sm_100a, loaded with cudaLibraryLoadData.
//
// Replaces the reference's pipeline construction (src/metal_backend.mm:233-560:
// load the library metallib and the user metallib, look the callables up by
// name, link them into the rollout pipelines through visible function
// tables).  Here the callables are bound by name at compile time, so they
// inline into the rollout kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace mppi_b200 {

struct ModuleSpec {
  std::string plugin_path;    // CUDA source of the callables
  std::string dynamics;       // required
  std::string stage_cost;     // "" = library default
  std::string terminal_cost;  // "" = library default
  uint32_t state_dim = 0;
  uint32_t control_dim = 0;
  bool cov_full = false;
  bool control_cost = false;
  bool noise_half = false;  // NumericMode kFp16 / kMixed: FP16 noise
  bool proposal = false;    // rollout reads a learned proposal (MPPI_PROPOSAL)
  std::string features;     // proposal-feature callable ("" = none)
  uint64_t model_params_bytes = 0;
  uint64_t cost_params_bytes = 0;
  // ParamLayout alignments and schema_hash, checked at compile time against
  // a plugin's MPPI_PARAM_LAYOUT declaration (mppi_prelude.cuh)
  uint64_t model_params_alignment = 1;
  uint64_t cost_params_alignment = 1;
  std::string schema_hash;
};

// Whether `s` can travel as the schema string of the compile (printable
// ASCII without quotes or backslashes, at most 256 characters).
bool valid_schema_hash(const std::string& s);

// Rollout block sizes compiled into every module (mppi_rollout_b<N>).
constexpr int kRolloutBlocks[3] = {64, 128, 256};

struct KernelModule {
  cudaLibrary_t library = nullptr;
  cudaKernel_t rollout[3] = {nullptr, nullptr, nullptr};
  cudaKernel_t rollout_work = nullptr;  // uneven batches (128-thread CTAs)
  // the same with each agent's combine run by its last CTA
  cudaKernel_t rollout_fused[3] = {nullptr, nullptr, nullptr};
  cudaKernel_t rollout_work_fused = nullptr;
  // warp-specialised 128-sample forms (256 threads), plain and fused
  // 128-sample forms with the early noise (whole horizon staged), plain and fused
  cudaKernel_t rollout_early = nullptr;
  cudaKernel_t rollout_early_fused = nullptr;
  cudaKernel_t rollout_ws = nullptr;
  cudaKernel_t rollout_ws_fused = nullptr;
  size_t ws_static_smem = 0;
  // cooperative forms (coop_lanes threads per sample), plain and fused:
  // [0] 32 samples per CTA (latency-bound launches), [1] 128 samples per CTA;
  // coop_lanes = 0 when the plugin declares no split stage cost
  cudaKernel_t rollout_coop[2] = {nullptr, nullptr};
  cudaKernel_t rollout_coop_fused[2] = {nullptr, nullptr};
  uint32_t coop_lanes = 0;
  size_t coop_static_smem[2] = {0, 0};
  cudaKernel_t combine = nullptr;
  cudaKernel_t weights = nullptr;
  cudaKernel_t noise = nullptr;
  cudaKernel_t features = nullptr;  // only when ModuleSpec::features is set
  // features + the per-agent network, one CTA per row (same condition)
  cudaKernel_t proposal_rows = nullptr;
  // static shared memory of the rollout kernels, the larger of the plain and
  // fused forms (their dynamic share is sized so that this plus the dynamic
  // part keeps the target residency)
  size_t rollout_static_smem[3] = {0, 0, 0};
  size_t work_static_smem = 0;
  std::string build_log;  // NVRTC log of the compile (warnings, ptxas info)
};

// Status codes mirror include/mppi_b200/mppi_backend.h.
// Returns 0 and a shared module (cached per process and, when a cache
// directory is usable, on disk) or an error code with a message.
int load_module(const ModuleSpec& spec, std::shared_ptr<const KernelModule>* out,
                std::string* error);

// Compiles the module without loading it (no GPU needed); `log` receives the
// NVRTC log including ptxas resource usage.
int compile_check(const ModuleSpec& spec, std::string* log, std::string* error);

// The embedded device sources (generated at build time).
const char* embedded_source(const char* name);

}  // namespace mppi_b200
