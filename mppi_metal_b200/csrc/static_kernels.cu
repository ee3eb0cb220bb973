// static_kernels.cu — kernels compiled ahead of time by nvcc for sm_100a
// (no plugin dependency): the Philox-2x32-10 known-answer path and the
// accuracy path of the library's own sine / cosine.
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/mppi_b200/mppi_backend.h"
#include "device/mppi_prelude.cuh"

namespace {

__global__ void __launch_bounds__(256)
    philox_words_kernel(uint64_t n, const uint32_t* c0, const uint32_t* c1, const uint32_t* key,
                        uint2* out) {
  const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  if (i < n) out[i] = mppi_philox2x32_10(make_uint2(c0[i], c1[i]), key[i]);
}

__global__ void __launch_bounds__(256)
    sincos_kernel(uint64_t n, const float* x, int quarter, float* so, float* co) {
  const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  float s, c;
  if (quarter)
    mppi_sincos_quarter(x[i], &s, &c);
  else
    mppi_sincosf(x[i], &s, &c);
  so[i] = s;
  co[i] = c;
}

__global__ void __launch_bounds__(256) log_kernel(uint64_t n, const float* x, float* out) {
  const uint64_t i = (uint64_t)blockIdx.x * 256 + threadIdx.x;
  if (i < n) out[i] = mppi_log(x[i]);
}

void set_err(char* err, size_t len, const std::string& msg) {
  if (err && len) {
    const size_t k = msg.size() < len - 1 ? msg.size() : len - 1;
    memcpy(err, msg.data(), k);
    err[k] = '\0';
  }
}

}  // namespace

extern "C" int mppi_device_philox(uint64_t n, const uint32_t* c0, const uint32_t* c1,
                                  const uint32_t* key, uint32_t* out, char* err,
                                  size_t err_len) {
  if (n == 0) return MPPI_OK;
  if (!c0 || !c1 || !key || !out) {
    set_err(err, err_len, "null argument to mppi_device_philox.");
    return MPPI_ERR_INVALID;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_err(err, err_len, "No CUDA device available.");
    return MPPI_ERR_NO_DEVICE;
  }
  void* buf = nullptr;
  const size_t in_bytes = n * 4;
  cudaError_t e = cudaMalloc(&buf, 3 * in_bytes + 2 * in_bytes);
  if (e == cudaSuccess) {
    // [out pairs 2n][c0 n][c1 n][key n]: the uint2 output sits at the
    // (256-byte aligned) base so every pair is 8-byte aligned.
    uint32_t* d = static_cast<uint32_t*>(buf);
    uint2* o = reinterpret_cast<uint2*>(d);
    uint32_t* dc0 = d + 2 * n;
    cudaMemcpy(dc0, c0, in_bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dc0 + n, c1, in_bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(dc0 + 2 * n, key, in_bytes, cudaMemcpyHostToDevice);
    philox_words_kernel<<<(unsigned)((n + 255) / 256), 256>>>(n, dc0, dc0 + n, dc0 + 2 * n, o);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(out, o, 2 * in_bytes, cudaMemcpyDeviceToHost);
    cudaFree(buf);
  }
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}

extern "C" int mppi_device_sincos(uint64_t n, const float* x, int quarter, float* sin_out,
                                  float* cos_out, char* err, size_t err_len) {
  if (n == 0) return MPPI_OK;
  if (!x || !sin_out || !cos_out) {
    set_err(err, err_len, "null argument to mppi_device_sincos.");
    return MPPI_ERR_INVALID;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_err(err, err_len, "No CUDA device available.");
    return MPPI_ERR_NO_DEVICE;
  }
  void* buf = nullptr;
  const size_t bytes = n * 4;
  cudaError_t e = cudaMalloc(&buf, 3 * bytes);
  if (e == cudaSuccess) {
    float* dx = static_cast<float*>(buf);  // [x n][sin n][cos n]
    e = cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      sincos_kernel<<<(unsigned)((n + 255) / 256), 256>>>(n, dx, quarter ? 1 : 0, dx + n,
                                                          dx + 2 * n);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(sin_out, dx + n, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(cos_out, dx + 2 * n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(buf);
  }
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}

extern "C" int mppi_device_log(uint64_t n, const float* x, float* out, char* err,
                               size_t err_len) {
  if (n == 0) return MPPI_OK;
  if (!x || !out) {
    set_err(err, err_len, "null argument to mppi_device_log.");
    return MPPI_ERR_INVALID;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_err(err, err_len, "No CUDA device available.");
    return MPPI_ERR_NO_DEVICE;
  }
  void* buf = nullptr;
  const size_t bytes = n * 4;
  cudaError_t e = cudaMalloc(&buf, 2 * bytes);
  if (e == cudaSuccess) {
    float* dx = static_cast<float*>(buf);  // [x n][out n]
    e = cudaMemcpy(dx, x, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      log_kernel<<<(unsigned)((n + 255) / 256), 256>>>(n, dx, dx + n);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dx + n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(buf);
  }
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}
