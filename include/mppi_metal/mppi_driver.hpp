// mppi_driver.hpp — the MPPI controller driver, B200 (CUDA) backend.
//
// Drop-in for the reference's include/mppi_metal/mppi_driver.hpp:18-96:
// same class, same methods, same bool + optional error-string convention,
// same lifecycle (construct -> initialize -> set_problem_params -> step ...).
// Overloads added by this project are marked; none changes an existing one.
#pragma once

#include "mppi_metal/mppi_types.hpp"

#include <memory>
#include <string>

namespace mppi_metal {

class MPPIDriver {
public:
	// Deep-copies sigma, sigma_inv, u_min and u_max (reference
	// mppi_driver.cpp:40-76).  No GPU work happens here.
	explicit MPPIDriver(const DriverConfig& config);
	// Added: the same, with options beyond the reference's method.
	MPPIDriver(const DriverConfig& config, const DriverOptions& options);
	~MPPIDriver();

	MPPIDriver(const MPPIDriver&) = delete;
	MPPIDriver& operator=(const MPPIDriver&) = delete;

	MPPIDriver(MPPIDriver&&) noexcept;
	MPPIDriver& operator=(MPPIDriver&&) noexcept;

	// Validates the config (hard-fail), compiles the plugin source with the
	// library kernels for sm_100a (NVRTC), loads them, allocates device state.
	bool initialize(const ModelPluginSpec& model, std::string* error = nullptr);

	// Copies the parameter blobs to device memory for reuse across steps.
	bool set_problem_params(const ProblemParams& params, std::string* error = nullptr);

	// Blocking: rollout -> weights -> update on the GPU; writes the updated
	// control sequence to u_next_out and the diagnostics, then warm-starts the
	// internal nominal (shift left, hold last) and advances the step index.
	bool step(
		const StepInputs& inputs,
		const MutableControlSequenceView& u_next_out,
		StepDiagnostics* diagnostics,
		std::string* error = nullptr
	);

	// Zeroes the internal nominal and the step index (as the reference's
	// implementation does).  Bound ProblemParams are kept.
	bool reset(std::string* error = nullptr);

	// Replaces the internal nominal (exact shape required); step index -> 0.
	bool reset(const ControlSequenceView& u_nominal, std::string* error = nullptr);

	// Closed loop of num_steps control steps on the GPU: the true state is
	// propagated with each step's first optimal control, the nominal is
	// warm-started on the device, and the history is returned.
	bool simulate(
		uint32_t num_steps,
		const StepInputs& initial_inputs,
		const SimulationResults& results,
		std::string* error = nullptr
	);

	// Closed loop for num_agents independent agents in one launch per pass;
	// agent a draws with key seed + a.  All agents start from a zero nominal.
	bool simulate_batch(
		uint32_t num_agents,
		uint32_t num_steps,
		const float* x0_packed,
		const BatchSimulationResults& results,
		std::string* error = nullptr
	);

	// Added: simulate_batch with per-agent parameter blobs and sigma.
	bool simulate_batch(
		uint32_t num_agents,
		uint32_t num_steps,
		const float* x0_packed,
		const BatchAgentParams& agent_params,
		const BatchSimulationResults& results,
		std::string* error = nullptr
	);

private:
	class Impl;
	std::unique_ptr<Impl> impl_;
};

}  // namespace mppi_metal
