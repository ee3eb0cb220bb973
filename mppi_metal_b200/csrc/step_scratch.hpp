// step_scratch.hpp — internal: one single-agent control step launched on
// caller-provided device memory plus a caller-provided scratch area
// (csrc/backend.cpp), used by the allocation-free entry point in
// csrc/noalloc.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>

struct mppi_backend;

namespace mppi_b200 {

// Floats of scratch one step needs for the backend's configuration
// (a zero word block, the per-CTA partials, the combine statistics).
size_t step_scratch_floats(const mppi_backend* b);

// Enqueues rollout + combine for one agent on `stream`.  Reads x0, u_nominal
// and the two parameter blobs from device memory, writes u_out and diag3 to
// device memory, and uses only `scratch` (device memory, >= the size above)
// for everything else.  Calls no allocating CUDA routine.
int launch_step_with_scratch(mppi_backend* b, uint64_t step_index, const float* x0,
                             const float* u_nominal, const void* model_params,
                             const void* cost_params, float* u_out, float* diag3,
                             float* scratch, size_t scratch_floats, cudaStream_t stream,
                             std::string* error);

// The backend's device and stream (for callers of the function above).
int backend_device(const mppi_backend* b);
cudaStream_t backend_stream(const mppi_backend* b);
bool backend_initialized(const mppi_backend* b);
// Whether a learned proposal network is attached (mppi_backend_set_proposal).
bool backend_has_proposal(const mppi_backend* b);

}  // namespace mppi_b200
