// noalloc.cu — the allocation-free single-agent control step.
//
// Who needs it: callers that must never allocate device memory once they are
// running -- a fixed-rate robot control loop, where cudaMalloc / cudaFree can
// stall for milliseconds and synchronise the whole device, or a host
// application whose device memory is owned by another framework's allocator
// and budgeted up front.  Such a caller keeps its own device buffers for the
// inputs and outputs and calls mppi_backend_dispatch_rollout_noalloc each
// control period; the temporary data of the step (the rollout blocks'
// partial sums and the combine statistics) lives in the fixed array below
// instead of in buffers the backend would otherwise allocate for the step.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// library holds MPPI_NOALLOC_SCRATCH_BYTES of it until the process exits.
// In host code its name is only a host-side stand-in, so the device address
// is looked up with cudaGetSymbolAddress, once per device, on that device's
// first call; that first call should therefore come before any stream
// capture.  The address is cached for the life of the process: a
// cudaDeviceReset while this library is in use is not supported (it also
// invalidates every backend's own buffers).  All calls share the one array
// and it keeps the previous call's contents (the entry point clears the part
// that must start at zero), so calls whose work overlaps on the GPU -- from
// two threads, or on two streams without ordering -- race on it.
//
// The step runs on the backend's own stream: the caller's inputs must be
// complete in device memory before the call (synchronise the stream that
// wrote them), and the outputs are complete when the call returns.  The
// caller's current device is restored before returning.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mppi_b200/mppi_backend.h"
#include "step_scratch.hpp"

namespace {

constexpr size_t kScratchFloats = MPPI_NOALLOC_SCRATCH_BYTES / sizeof(float);

// The step's scratch: zero block, per-CTA partial records, statistics.
static __device__ __align__(256) float g_step_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_lookup_mutex;
float* g_scratch_addr[kMaxDevices] = {nullptr};

void put_err(char* err, size_t len, const std::string& msg) {
  if (err && len) {
    const size_t n = msg.size() < len - 1 ? msg.size() : len - 1;
    memcpy(err, msg.data(), n);
    err[n] = '\0';
  }
}

// Makes `dev` current for the lifetime of the object and restores the
// caller's device afterwards.
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int dev) {
    status = cudaGetDevice(&prev);
    if (status == cudaSuccess && prev != dev) status = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" int mppi_backend_dispatch_rollout_noalloc(
    mppi_backend* b, uint64_t step_index, const float* x0, const float* u_nominal,
    const void* model_params, const void* cost_params, float* u_out, float* diag3, char* err,
    size_t err_len) {
  if (!mppi_b200::backend_initialized(b)) {
    put_err(err, err_len, "MPPI backend is not initialized.");
    return MPPI_ERR_NOT_INIT;
  }
  if (!x0 || !u_nominal || !u_out || !diag3) {
    put_err(err, err_len, "x0, u_nominal, u_out and diag3 must be device pointers, not null.");
    return MPPI_ERR_INVALID;
  }
  if (mppi_b200::backend_has_proposal(b)) {
    put_err(err, err_len,
            "mppi_backend_dispatch_rollout_noalloc: a learned proposal network is attached; "
            "this entry point runs plain MPPI only (detach it with mppi_backend_set_proposal("
            "b, NULL, 0, ...) or use mppi_backend_dispatch_rollout).");
    return MPPI_ERR_INVALID;
  }
  const size_t need = mppi_b200::step_scratch_floats(b);
  if (need > kScratchFloats) {
    put_err(err, err_len,
            "mppi_backend_dispatch_rollout_noalloc: this problem needs " +
                std::to_string(need * sizeof(float)) + " bytes of scratch, more than the " +
                std::to_string(MPPI_NOALLOC_SCRATCH_BYTES) +
                "-byte static area (reduce sample_count or horizon * control_dim, or use "
                "mppi_backend_dispatch_rollout).");
    return MPPI_ERR_INVALID;
  }
  const int dev = mppi_b200::backend_device(b);
  if (dev < 0 || dev >= kMaxDevices) {
    put_err(err, err_len, "device ordinal out of range.");
    return MPPI_ERR_INVALID;
  }
  DeviceGuard guard(dev);
  if (guard.status != cudaSuccess) {
    put_err(err, err_len, std::string("cudaSetDevice: ") + cudaGetErrorString(guard.status));
    return MPPI_ERR_CUDA;
  }
  float* scratch = nullptr;
  {
    // one-time set-up per device, with that device current
    std::lock_guard<std::mutex> lock(g_lookup_mutex);
    if (g_scratch_addr[dev] == nullptr) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
      if (e != cudaSuccess || p == nullptr) {
        put_err(err, err_len, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                  cudaGetErrorString(e));
        return MPPI_ERR_CUDA;
      }
      g_scratch_addr[dev] = static_cast<float*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  cudaStream_t s = mppi_b200::backend_stream(b);
  std::string msg;
  int rc = mppi_b200::launch_step_with_scratch(b, step_index, x0, u_nominal, model_params,
                                               cost_params, u_out, diag3, scratch,
                                               kScratchFloats, s, &msg);
  if (rc != MPPI_OK) {
    put_err(err, err_len, msg);
    return rc;
  }
  const cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    put_err(err, err_len, std::string("step failed: ") + cudaGetErrorString(e));
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}
