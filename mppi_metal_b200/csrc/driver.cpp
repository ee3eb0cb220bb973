// driver.cpp — mppi_metal::MPPIDriver on the CUDA backend.
//
// Same semantics as the reference's src/mppi_driver.cpp (validation order and
// messages, warm start, step-index bookkeeping, batch zero nominal); the
// backend behind it is the C ABI of include/mppi_b200/mppi_backend.h instead
// of MetalBackend.  Hardening beyond the reference is marked "added".
#include "mppi_metal/mppi_driver.hpp"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mppi_b200/mppi_backend.h"
#include "proposal.hpp"

namespace mppi_metal {

namespace {

constexpr size_t kErrLen = 8192;

bool is_pow2(size_t v) { return v != 0 && (v & (v - 1)) == 0; }

}  // namespace

class MPPIDriver::Impl {
public:
	Impl(const DriverConfig& cfg, const DriverOptions& opts);
	~Impl() {
		if (backend) mppi_backend_destroy(backend);
	}

	DriverConfig config;
	DriverOptions options;
	std::vector<float> sigma_storage;
	std::vector<float> sigma_inv_storage;
	std::vector<float> u_min_storage;
	std::vector<float> u_max_storage;
	std::vector<float> u_nominal;  // horizon * control_dim warm start
	std::string proposal_features;  // owned copy of options.proposal_features
	std::vector<float> u_updated;   // step(): the updated sequence (reused, no per-step allocation)
	std::vector<char> step_err;     // step(): error text buffer (reused)

	ParamLayout param_layout{};
	bool params_bound = false;

	mppi_backend* backend = nullptr;
	bool initialized = false;
	uint64_t step_index = 0;
};

// Deep copies (reference mppi_driver.cpp:40-76): sigma / sigma_inv hold m
// floats for kDiagonal, m*m for kFull; bounds hold m floats.
MPPIDriver::Impl::Impl(const DriverConfig& cfg, const DriverOptions& opts)
	: config(cfg), options(opts), proposal_features(opts.proposal_features) {
	options.proposal_features = proposal_features;  // the caller's view need not outlive us
	const uint32_t m = cfg.control_dim;
	const size_t nsig = cfg.noise.covariance_form == ControlNoiseConfig::CovarianceForm::kDiagonal
		? m
		: static_cast<size_t>(m) * m;
	if (cfg.noise.sigma != nullptr && m > 0) {
		sigma_storage.assign(cfg.noise.sigma, cfg.noise.sigma + nsig);
		config.noise.sigma = sigma_storage.data();
	}
	if (cfg.noise.sigma_inv != nullptr && m > 0) {
		sigma_inv_storage.assign(cfg.noise.sigma_inv, cfg.noise.sigma_inv + nsig);
		config.noise.sigma_inv = sigma_inv_storage.data();
	}
	if (cfg.bounds.u_min != nullptr && m > 0) {
		u_min_storage.assign(cfg.bounds.u_min, cfg.bounds.u_min + m);
		config.bounds.u_min = u_min_storage.data();
	}
	if (cfg.bounds.u_max != nullptr && m > 0) {
		u_max_storage.assign(cfg.bounds.u_max, cfg.bounds.u_max + m);
		config.bounds.u_max = u_max_storage.data();
	}
	u_nominal.assign(static_cast<size_t>(cfg.horizon) * cfg.control_dim, 0.0f);
}

MPPIDriver::MPPIDriver(const DriverConfig& config)
	: impl_(std::make_unique<Impl>(config, DriverOptions{})) {}

MPPIDriver::MPPIDriver(const DriverConfig& config, const DriverOptions& options)
	: impl_(std::make_unique<Impl>(config, options)) {}

MPPIDriver::~MPPIDriver() = default;
MPPIDriver::MPPIDriver(MPPIDriver&&) noexcept = default;
MPPIDriver& MPPIDriver::operator=(MPPIDriver&&) noexcept = default;

bool MPPIDriver::initialize(const ModelPluginSpec& model, std::string* error) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	const auto& cfg = impl_->config;

	// ---- dimensions (reference mppi_driver.cpp:100-116) ----
	if (cfg.state_dim == 0) return fail("DriverConfig::state_dim must be > 0.");
	if (cfg.control_dim == 0) return fail("DriverConfig::control_dim must be > 0.");
	if (cfg.horizon == 0) return fail("DriverConfig::horizon must be > 0.");
	if (cfg.sample_count == 0) return fail("DriverConfig::sample_count must be > 0.");

	// ---- noise (reference :118-133) ----
	if (cfg.noise.control_dim != cfg.control_dim) {
		return fail("ControlNoiseConfig::control_dim (" + std::to_string(cfg.noise.control_dim) +
			") must match DriverConfig::control_dim (" + std::to_string(cfg.control_dim) + ").");
	}
	if (cfg.noise.sigma == nullptr) return fail("ControlNoiseConfig::sigma must not be null.");
	if (cfg.noise.sigma_inv == nullptr) return fail("ControlNoiseConfig::sigma_inv must not be null.");

	// ---- bounds (reference :135-159) ----
	if (cfg.bounds.control_dim != cfg.control_dim) {
		return fail("ControlBounds::control_dim (" + std::to_string(cfg.bounds.control_dim) +
			") must match DriverConfig::control_dim (" + std::to_string(cfg.control_dim) + ").");
	}
	if (cfg.bounds.u_min == nullptr)
		return fail("ControlBounds::u_min must not be null when control_dim > 0.");
	if (cfg.bounds.u_max == nullptr)
		return fail("ControlBounds::u_max must not be null when control_dim > 0.");
	for (uint32_t i = 0; i < cfg.bounds.control_dim; ++i) {
		if (cfg.bounds.u_min[i] > cfg.bounds.u_max[i]) {
			return fail("ControlBounds::u_min[" + std::to_string(i) + "] (" +
				std::to_string(cfg.bounds.u_min[i]) + ") > u_max[" + std::to_string(i) + "] (" +
				std::to_string(cfg.bounds.u_max[i]) + ").");
		}
	}

	// ---- added: the limits the reference's kernels silently truncate at
	// (shaders/mppi_core.h:32-33; the state buffer is sized per module here,
	// up to MPPI_MAX_STATE_DIM floats), and the ParamLayout alignment
	// contract ----
	if (cfg.state_dim > MPPI_MAX_STATE_DIM) {
		return fail("DriverConfig::state_dim (" + std::to_string(cfg.state_dim) +
			") exceeds the state limit of " + std::to_string(MPPI_MAX_STATE_DIM) + " floats.");
	}
	if (cfg.control_dim > 16u) {
		return fail("DriverConfig::control_dim (" + std::to_string(cfg.control_dim) +
			") exceeds the control limit of 16.");
	}
	if (!is_pow2(model.param_layout.model_params_alignment))
		return fail("ParamLayout::model_params_alignment must be a power of two.");
	if (!is_pow2(model.param_layout.cost_params_alignment))
		return fail("ParamLayout::cost_params_alignment must be a power of two.");

	// ---- backend: compile plugin + kernels, allocate (reference :161-164) ----
	if (impl_->backend) {
		mppi_backend_destroy(impl_->backend);
		impl_->backend = nullptr;
		impl_->initialized = false;
	}
	if (mppi_backend_create(&impl_->backend) != MPPI_OK) return fail("out of memory creating the backend.");
	const std::string path = model.user_metallib_path.string();
	const std::string dyn(model.callables.dynamics);
	const std::string stage(model.callables.stage_cost);
	const std::string term(model.callables.terminal_cost);
	mppi_backend_plugin plug{};
	plug.source_path = path.c_str();
	plug.dynamics = dyn.c_str();
	plug.stage_cost = stage.c_str();
	plug.terminal_cost = term.c_str();
	plug.model_params_size = model.param_layout.model_params_size;
	plug.cost_params_size = model.param_layout.cost_params_size;
	plug.seed = model.rng.seed;
	plug.model_params_alignment = model.param_layout.model_params_alignment;
	plug.cost_params_alignment = model.param_layout.cost_params_alignment;
	plug.schema_hash = model.param_layout.schema_hash.c_str();
	mppi_backend_config bc{};
	bc.state_dim = cfg.state_dim;
	bc.control_dim = cfg.control_dim;
	bc.horizon = cfg.horizon;
	bc.sample_count = cfg.sample_count;
	bc.lambda = cfg.lambda;
	bc.covariance_form = cfg.noise.covariance_form == ControlNoiseConfig::CovarianceForm::kFull ? 1u : 0u;
	bc.sigma = cfg.noise.sigma;
	bc.sigma_inv = cfg.noise.sigma_inv;
	bc.u_min = cfg.bounds.u_min;
	bc.u_max = cfg.bounds.u_max;
	bc.numeric_mode = static_cast<uint32_t>(cfg.numeric_mode);
	bc.control_cost = impl_->options.control_cost ? 1u : 0u;
	std::vector<char> err(kErrLen, '\0');
	if (mppi_backend_initialize(impl_->backend, &plug, &bc, err.data(), err.size()) != MPPI_OK) {
		mppi_backend_destroy(impl_->backend);
		impl_->backend = nullptr;
		return fail(err.data());
	}

	if (impl_->options.proposal != nullptr) {
		const mppi_b200::ProposalShape ps = mppi_b200::proposal_shape(impl_->options.proposal);
		const std::string& feat = impl_->proposal_features;
		if (mppi_backend_set_features(impl_->backend, feat.c_str(), ps.input_dim, err.data(),
		                              err.size()) != MPPI_OK ||
		    mppi_backend_set_proposal(impl_->backend, impl_->options.proposal,
		                              impl_->options.proposal_samples, err.data(),
		                              err.size()) != MPPI_OK) {
			mppi_backend_destroy(impl_->backend);
			impl_->backend = nullptr;
			return fail(err.data());
		}
	}

	impl_->param_layout = model.param_layout;
	impl_->params_bound = false;
	impl_->initialized = true;
	return true;
}

bool MPPIDriver::set_problem_params(const ProblemParams& params, std::string* error) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	if (!impl_->initialized) return fail("Driver is not initialized. Call initialize() first.");
	const auto& layout = impl_->param_layout;

	// ---- model params (reference mppi_driver.cpp:186-204) ----
	if (layout.model_params_size > 0 && params.model_params.bytes == 0) {
		return fail("ParamLayout declares model_params_size " + std::to_string(layout.model_params_size) +
			" but provided model_params.bytes is 0.");
	}
	if (params.model_params.bytes > 0 && params.model_params.bytes != layout.model_params_size) {
		return fail("model_params.bytes (" + std::to_string(params.model_params.bytes) +
			") does not match ParamLayout::model_params_size (" +
			std::to_string(layout.model_params_size) + ").");
	}
	if (params.model_params.bytes > 0 && params.model_params.data == nullptr)
		return fail("model_params.data is null but bytes > 0.");

	// ---- cost params (reference :206-224) ----
	if (layout.cost_params_size > 0 && params.cost_params.bytes == 0) {
		return fail("ParamLayout declares cost_params_size " + std::to_string(layout.cost_params_size) +
			" but provided cost_params.bytes is 0.");
	}
	if (params.cost_params.bytes > 0 && params.cost_params.bytes != layout.cost_params_size) {
		return fail("cost_params.bytes (" + std::to_string(params.cost_params.bytes) +
			") does not match ParamLayout::cost_params_size (" +
			std::to_string(layout.cost_params_size) + ").");
	}
	if (params.cost_params.bytes > 0 && params.cost_params.data == nullptr)
		return fail("cost_params.data is null but bytes > 0.");

	// ---- added: declared alignment (README "Hard-fail validation rules") ----
	if (params.model_params.bytes > 0 &&
		reinterpret_cast<uintptr_t>(params.model_params.data) % layout.model_params_alignment != 0)
		return fail("model_params.data is not aligned to ParamLayout::model_params_alignment.");
	if (params.cost_params.bytes > 0 &&
		reinterpret_cast<uintptr_t>(params.cost_params.data) % layout.cost_params_alignment != 0)
		return fail("cost_params.data is not aligned to ParamLayout::cost_params_alignment.");

	std::vector<char> err(kErrLen, '\0');
	if (mppi_backend_bind_params(impl_->backend, params.model_params.data, params.model_params.bytes,
			params.cost_params.data, params.cost_params.bytes, err.data(), err.size()) != MPPI_OK)
		return fail(err.data());
	impl_->params_bound = true;
	return true;
}

bool MPPIDriver::step(
	const StepInputs& inputs,
	const MutableControlSequenceView& u_next_out,
	StepDiagnostics* diagnostics,
	std::string* error
) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	// ---- reference mppi_driver.cpp:247-289 ----
	if (!impl_->initialized) return fail("Driver is not initialized. Call initialize() first.");
	const auto& cfg = impl_->config;
	if (inputs.x0.data == nullptr) return fail("StepInputs::x0.data must not be null.");
	if (inputs.x0.state_dim != cfg.state_dim) {
		return fail("StepInputs::x0.state_dim (" + std::to_string(inputs.x0.state_dim) +
			") must match DriverConfig::state_dim (" + std::to_string(cfg.state_dim) + ").");
	}
	if (u_next_out.data == nullptr) return fail("u_next_out.data must not be null.");
	if (u_next_out.horizon != cfg.horizon || u_next_out.control_dim != cfg.control_dim)
		return fail("u_next_out shape mismatch.");
	const float* active_nominal = impl_->u_nominal.data();
	if (inputs.u_nominal_override.data != nullptr) {
		if (inputs.u_nominal_override.horizon != cfg.horizon ||
			inputs.u_nominal_override.control_dim != cfg.control_dim)
			return fail("u_nominal_override shape mismatch.");
		active_nominal = inputs.u_nominal_override.data;
	}

	// ---- dispatch (reference :291-321); bytes == 0 selects the bound blob ----
	const size_t seq = static_cast<size_t>(cfg.horizon) * cfg.control_dim;
	std::vector<float>& u_updated = impl_->u_updated;
	u_updated.resize(seq);
	float diag[3] = {0.0f, 0.0f, 0.0f};
	std::vector<char>& err = impl_->step_err;
	if (err.size() != kErrLen) err.assign(kErrLen, '\0');
	err[0] = '\0';
	const ByteView& mo = inputs.model_params_override;
	const ByteView& co = inputs.cost_params_override;
	if (mppi_backend_dispatch_rollout(impl_->backend, impl_->step_index, inputs.x0.data,
			active_nominal, mo.bytes > 0 ? mo.data : nullptr, mo.bytes,
			co.bytes > 0 ? co.data : nullptr, co.bytes, u_updated.data(), diag, err.data(),
			err.size()) != MPPI_OK)
		return fail(err.data());
	if (diagnostics != nullptr) {
		diagnostics->best_cost = diag[0];
		diagnostics->mean_cost = diag[1];
		diagnostics->effective_sample_size = diag[2];
		diagnostics->converged = false;
	}

	// ---- output + warm start: shift left, hold last (reference :323-339) ----
	std::copy(u_updated.begin(), u_updated.end(), u_next_out.data);
	const uint32_t m = cfg.control_dim, H = cfg.horizon;
	for (uint32_t t = 0; t + 1 < H; ++t)
		for (uint32_t d = 0; d < m; ++d) impl_->u_nominal[t * m + d] = u_updated[(t + 1) * m + d];
	for (uint32_t d = 0; d < m; ++d) impl_->u_nominal[(H - 1) * m + d] = u_updated[(H - 1) * m + d];
	++impl_->step_index;
	return true;
}

bool MPPIDriver::simulate(
	uint32_t num_steps,
	const StepInputs& inputs,
	const SimulationResults& results,
	std::string* error
) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	// ---- reference mppi_driver.cpp:355-403 ----
	if (!impl_->initialized) return fail("Driver is not initialized. Call initialize() first.");
	if (num_steps == 0) return fail("num_steps must be > 0.");
	const auto& cfg = impl_->config;
	if (inputs.x0.data == nullptr) return fail("StepInputs::x0.data must not be null.");
	if (inputs.x0.state_dim != cfg.state_dim) {
		return fail("StepInputs::x0.state_dim (" + std::to_string(inputs.x0.state_dim) +
			") must match DriverConfig::state_dim (" + std::to_string(cfg.state_dim) + ").");
	}
	if (results.num_steps != num_steps) return fail("SimulationResults::num_steps mismatch.");
	const float* active_nominal = impl_->u_nominal.data();
	if (inputs.u_nominal_override.data != nullptr) {
		if (inputs.u_nominal_override.horizon != cfg.horizon ||
			inputs.u_nominal_override.control_dim != cfg.control_dim)
			return fail("u_nominal_override shape mismatch.");
		active_nominal = inputs.u_nominal_override.data;
	}
	const ByteView& mo = inputs.model_params_override;
	const ByteView& co = inputs.cost_params_override;
	std::vector<char> err(kErrLen, '\0');
	if (mppi_backend_dispatch_simulation(impl_->backend, num_steps, impl_->step_index,
			inputs.x0.data, active_nominal, mo.bytes > 0 ? mo.data : nullptr, mo.bytes,
			co.bytes > 0 ? co.data : nullptr, co.bytes, results.states_out, results.controls_out,
			results.costs_out, err.data(), err.size()) != MPPI_OK)
		return fail(err.data());
	impl_->step_index += num_steps;  // reference :419
	return true;
}

bool MPPIDriver::simulate_batch(
	uint32_t num_agents,
	uint32_t num_steps,
	const float* x0_packed,
	const BatchSimulationResults& results,
	std::string* error
) {
	return simulate_batch(num_agents, num_steps, x0_packed, BatchAgentParams{}, results, error);
}

bool MPPIDriver::simulate_batch(
	uint32_t num_agents,
	uint32_t num_steps,
	const float* x0_packed,
	const BatchAgentParams& agent_params,
	const BatchSimulationResults& results,
	std::string* error
) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	// ---- reference mppi_driver.cpp:436-463 ----
	if (!impl_->initialized) return fail("Driver is not initialized. Call initialize() first.");
	if (num_agents == 0) return fail("num_agents must be > 0.");
	if (num_steps == 0) return fail("num_steps must be > 0.");
	if (x0_packed == nullptr) return fail("x0_packed must not be null.");
	if (results.num_agents != num_agents) return fail("BatchSimulationResults::num_agents mismatch.");
	if (results.num_steps != num_steps) return fail("BatchSimulationResults::num_steps mismatch.");
	const auto& layout = impl_->param_layout;
	// added: per-agent blob strides must hold a whole ParamLayout blob
	if (agent_params.model_params != nullptr && num_agents > 1 &&
		agent_params.model_params_stride < layout.model_params_size)
		return fail("BatchAgentParams::model_params_stride is smaller than ParamLayout::model_params_size.");
	if (agent_params.cost_params != nullptr && num_agents > 1 &&
		agent_params.cost_params_stride < layout.cost_params_size)
		return fail("BatchAgentParams::cost_params_stride is smaller than ParamLayout::cost_params_size.");

	// Every agent starts from a zero nominal; overrides are not used
	// (reference :465-472).
	mppi_batch_agents ag{};
	ag.model_params = agent_params.model_params;
	ag.model_params_stride = agent_params.model_params_stride;
	ag.cost_params = agent_params.cost_params;
	ag.cost_params_stride = agent_params.cost_params_stride;
	ag.sigma = agent_params.sigma;
	ag.sample_counts = agent_params.sample_counts;
	ag.horizons = agent_params.horizons;
	const bool any = ag.model_params || ag.cost_params || ag.sigma || ag.sample_counts ||
		ag.horizons;
	std::vector<char> err(kErrLen, '\0');
	if (mppi_backend_dispatch_batch_simulation(impl_->backend, num_agents, num_steps,
			impl_->step_index, x0_packed, nullptr, any ? &ag : nullptr, results.states_out,
			results.controls_out, results.costs_out, results.terminal_states_out, err.data(),
			err.size()) != MPPI_OK)
		return fail(err.data());
	impl_->step_index += num_steps;  // reference :489
	return true;
}

// Zeroes the nominal and the step index (reference mppi_driver.cpp:493-500;
// the step index restarts at 0 there too, although its header says the RNG
// "continues").
bool MPPIDriver::reset(std::string* /*error*/) {
	std::fill(impl_->u_nominal.begin(), impl_->u_nominal.end(), 0.0f);
	impl_->step_index = 0;
	return true;
}

bool MPPIDriver::reset(const ControlSequenceView& u_nominal, std::string* error) {
	auto fail = [&](const std::string& msg) {
		if (error != nullptr) *error = msg;
		return false;
	};
	// ---- reference mppi_driver.cpp:509-536 ----
	const auto& cfg = impl_->config;
	if (u_nominal.horizon != cfg.horizon) {
		return fail("reset: u_nominal.horizon (" + std::to_string(u_nominal.horizon) +
			") must match DriverConfig::horizon (" + std::to_string(cfg.horizon) + ").");
	}
	if (u_nominal.control_dim != cfg.control_dim) {
		return fail("reset: u_nominal.control_dim (" + std::to_string(u_nominal.control_dim) +
			") must match DriverConfig::control_dim (" + std::to_string(cfg.control_dim) + ").");
	}
	const size_t n = static_cast<size_t>(cfg.horizon) * cfg.control_dim;
	if (n > 0 && u_nominal.data == nullptr)
		return fail("reset: u_nominal.data must not be null when horizon * control_dim > 0.");
	if (n > 0) std::copy(u_nominal.data, u_nominal.data + n, impl_->u_nominal.begin());
	impl_->step_index = 0;
	return true;
}

}  // namespace mppi_metal
