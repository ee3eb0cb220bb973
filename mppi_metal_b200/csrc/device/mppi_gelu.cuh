// mppi_gelu.cuh — the proposal network's activation, shared by its
// tensor-core kernels (csrc/proposal_mlp.cu, nvcc) and the per-agent network
// evaluation inside the MPPI module (mppi_kernels.cuh, NVRTC), so both
// compute the same GELU.
//
// GELU(z) = z Phi(z) with Phi(z) = (1 + erf(z / sqrt 2)) / 2, and its
// derivative Phi(z) + z phi(z).  erf by Abramowitz and Stegun, "Handbook of
// Mathematical Functions", eq. 7.1.26 (Hastings' approximation): for x >= 0,
// erf x = 1 - t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2) with
// t = 1 / (1 + p x), |error| <= 1.5e-7; the reciprocal and the exponential
// come from the SM's approximate instructions (relative errors of order
// 2^-22).  The exp(-x^2) = exp(-z^2 / 2) it computes is the Gaussian factor of
// the derivative as well.  The activations are rounded to BF16 (8 significant
// bits) before they feed the next layer, far above this error.
#pragma once

__device__ __forceinline__ void mppi_gelu_phi(float z, float& cdf, float& gauss) {
  const float x = fabsf(z) * 0.70710678118654752f;
  float t;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(t) : "f"(fmaf(0.3275911f, x, 1.0f)));
  float p = fmaf(1.061405429f, t, -1.453152027f);
  p = fmaf(p, t, 1.421413741f);
  p = fmaf(p, t, -0.284496736f);
  p = fmaf(p, t, 0.254829592f);
  p *= t;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(gauss) : "f"(-1.44269504088896341f * x * x));
  cdf = fmaf(0.5f, copysignf(fmaf(-p, gauss, 1.0f), z), 0.5f);
}

__device__ __forceinline__ float mppi_gelu(float z) {
  float cdf, g;
  mppi_gelu_phi(z, cdf, g);
  return z * cdf;
}

// Round to the nearest BF16 (ties to even), returned as the float it is.
__device__ __forceinline__ float mppi_round_bf16(float x) {
  unsigned short h;
  asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(h) : "f"(x));
  return __uint_as_float((unsigned)h << 16);
}
