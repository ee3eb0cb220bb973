// mppi_types.hpp — public configuration, plugin, view and result types.
//
// Drop-in for the reference's include/mppi_metal/mppi_types.hpp: every type,
// field name, field order and default below matches the reference
// (MarshallVielmetti/mppi_metal, include/mppi_metal/mppi_types.hpp:15-188) so
// code written against it recompiles unchanged.  Meaning changes on this
// backend are noted on the field.  Types added by this project sit at the end
// (DriverOptions, BatchAgentParams) and change none of the reference types.
#pragma once

#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <string>
#include <string_view>

struct mppi_proposal;  // include/mppi_b200/mppi_proposal.h

namespace mppi_metal {

// ---- control noise (reference mppi_types.hpp:15-29) ------------------------
struct ControlNoiseConfig {
	enum class CovarianceForm {
		kDiagonal,
		kFull
	};

	CovarianceForm covariance_form = CovarianceForm::kDiagonal;

	// kDiagonal: control_dim per-dimension standard deviations
	//            (noise_d = n_d * sigma[d], as the reference's kernels use it).
	// kFull:     control_dim * control_dim row-major covariance Sigma; the
	//            noise is L n with L its Cholesky factor.  (The reference
	//            accepts kFull but its kernels read only sigma[0..m).)
	const float* sigma = nullptr;
	// Sigma^-1 in the same form; used by DriverOptions::control_cost.
	const float* sigma_inv = nullptr;
	uint32_t control_dim = 0;
};

// ---- actuator limits (reference mppi_types.hpp:35-40) ----------------------
struct ControlBounds {
	const float* u_min = nullptr;  // control_dim elements
	const float* u_max = nullptr;  // control_dim elements
	uint32_t control_dim = 0;
};

// ---- driver configuration (reference mppi_types.hpp:46-62) ----------------
struct DriverConfig {
	uint32_t state_dim = 0;
	uint32_t control_dim = 0;
	uint32_t horizon = 0;
	uint32_t sample_count = 0;
	float lambda = 1.0f;
	ControlNoiseConfig noise;
	ControlBounds bounds;

	enum class NumericMode {
		kFp32,
		kFp16,
		kMixed
	};

	// kFp32: every value in FP32 (bit-exact Philox, accurate Box-Muller).
	// kFp16 / kMixed: the noise is drawn with approximate transcendentals and
	// rounded once to FP16, and that value is used by rollout and update
	// alike; the plugin's dynamics and costs, the weights and the update stay
	// FP32.  (The reference accepts the field and ignores it.)
	NumericMode numeric_mode = NumericMode::kFp32;
};

// ---- RNG (reference mppi_types.hpp:68-73) ---------------------------------
// Philox-2x32-10, counter = (step index, trajectory-derived id); the device
// key is the low 32 bits of seed (plus the agent index in batches).
struct RngConfig {
	uint64_t seed = 0;
};

// ---- model plugin (reference mppi_types.hpp:79-101) ------------------------
struct CallableNames {
	// Required __device__ dynamics function of the plugin source.
	std::string_view dynamics = "mppi_dynamics";
	// Optional cost functions; empty selects the library default (zero).
	std::string_view stage_cost = "";
	std::string_view terminal_cost = "";
};

struct ParamLayout {
	size_t model_params_size = 0;
	size_t model_params_alignment = 1;
	size_t cost_params_size = 0;
	size_t cost_params_alignment = 1;
	std::string schema_hash;
};

struct ModelPluginSpec {
	// On this backend: path of a CUDA source file defining the callables as
	// __device__ functions (compiled with NVRTC into the rollout kernel).
	// The name is kept for source compatibility.
	std::filesystem::path user_metallib_path;
	CallableNames callables;
	ParamLayout param_layout;
	RngConfig rng;
};

// ---- views (reference mppi_types.hpp:107-127) -----------------------------
struct StateView {
	const float* data = nullptr;
	uint32_t state_dim = 0;
};

struct ControlSequenceView {
	const float* data = nullptr;
	uint32_t horizon = 0;
	uint32_t control_dim = 0;
};

struct MutableControlSequenceView {
	float* data = nullptr;
	uint32_t horizon = 0;
	uint32_t control_dim = 0;
};

struct ByteView {
	const void* data = nullptr;
	size_t bytes = 0;
};

// ---- params and step inputs (reference mppi_types.hpp:133-150) -------------
struct ProblemParams {
	ByteView model_params;
	ByteView cost_params;
};

struct StepInputs {
	StateView x0;
	// Optional per-step nominal override (data == nullptr: internal warm start).
	ControlSequenceView u_nominal_override;
	// Optional per-step param overrides (bytes == 0: bound params).
	ByteView model_params_override;
	ByteView cost_params_override;
};

// ---- diagnostics (reference mppi_types.hpp:156-161) -------------------------
struct StepDiagnostics {
	float best_cost = 0.0f;
	float mean_cost = 0.0f;
	float effective_sample_size = 0.0f;
	bool converged = false;  // always false, as in the reference
};

// ---- simulation outputs (reference mppi_types.hpp:167-188) ------------------
struct SimulationResults {
	float* states_out = nullptr;     // [num_steps][state_dim]
	float* controls_out = nullptr;   // [num_steps][control_dim] (u*[0] of each step)
	float* costs_out = nullptr;      // [num_steps] best cost of each step
	uint32_t num_steps = 0;
};

// Histories are step-major: [step][agent][dim].
struct BatchSimulationResults {
	float* states_out = nullptr;          // [num_steps][num_agents][state_dim]
	float* controls_out = nullptr;        // [num_steps][num_agents][control_dim]
	float* costs_out = nullptr;           // [num_steps][num_agents]
	float* terminal_states_out = nullptr; // [num_agents][state_dim], after the last step
	uint32_t num_agents = 0;
	uint32_t num_steps = 0;
};

// ===========================================================================
// Additions of this project (no reference counterpart)
// ===========================================================================

// Options that change the method beyond the reference's; all default to the
// reference's behaviour.
struct DriverOptions {
	// Add lambda * u_nom_t^T Sigma^-1 eps_t to every stage cost (the MPPI
	// control-cost term of Williams et al.); Sigma^-1 is noise.sigma_inv.
	bool control_cost = false;

	// Learned sampling proposal (include/mppi_b200/mppi_proposal.h).  When
	// `proposal` is set, initialize() compiles the plugin's feature callable
	// `proposal_features` and every step draws `proposal_samples` of its
	// samples around the network's predicted sequence (the rest as plain
	// MPPI).  The caller owns the network and keeps it alive.
	struct mppi_proposal* proposal = nullptr;
	uint32_t proposal_samples = 0;
	std::string_view proposal_features = "mppi_proposal_features";
};

// Per-agent inputs for simulate_batch: every agent may carry its own model /
// cost parameter blob (ParamLayout-sized, `stride` bytes apart) and its own
// noise sigma (control_dim floats, or control_dim^2 for kFull).  Null
// pointers fall back to the bound ProblemParams / DriverConfig sigma.
struct BatchAgentParams {
	const void* model_params = nullptr;
	size_t model_params_stride = 0;
	const void* cost_params = nullptr;
	size_t cost_params_stride = 0;
	const float* sigma = nullptr;
	// Uneven batches: per-agent sample count (1..sample_count) and horizon
	// (1..horizon).  Null = the DriverConfig value for every agent.  An uneven
	// batch runs as one persistent launch per pass; its grid size and noise
	// staging are tuned on the first run of each shape without changing any
	// result.
	const uint32_t* sample_counts = nullptr;
	const uint32_t* horizons = nullptr;
};

}  // namespace mppi_metal
