// mppi_prelude.cuh — device-side basics shared by every kernel of the library
// and by user model plugins.
//
// Compiled two ways:
//   * by NVRTC, as the first part of the per-driver translation unit
//     (prelude + user plugin + mppi_kernels.cuh), see csrc/nvrtc_module.cpp;
//   * by nvcc, inside csrc/static_kernels.cu (Philox known-answer kernels).
//
// Contents
//   - fixed-width integer types under NVRTC (no libc headers there);
//   - the plugin callable ABI: the CUDA form of the reference's
//     shaders/mppi_core.h:11-42 (same argument order and meaning; the
//     reference's `thread` / `device` address spaces become plain pointers);
//   - Philox-2x32-10, the uint -> (0,1) map and Box-Muller, the CUDA form of
//     shaders/philox.h:19-50.  Words are bit-exact with the reference.  The
//     normals use correctly-rounded float ops for the uniform map (identical
//     bits to the reference), the library's own logarithm and quarter-turn
//     sine / cosine and the SM's square root (errors of order 1e-7);
//   - mppi_sincosf, the library's own sin / cos for plugins.
#pragma once

#if defined(__CUDACC_RTC__)
typedef unsigned char uint8_t;
typedef signed char int8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef unsigned long long uint64_t;
typedef long long int64_t;
#else
#include <cstdint>
#endif

#ifndef MPPI_MAX_STATE_BYTES
// Thread-local state buffer size (shaders/mppi_core.h:32: 128 bytes).  The
// library compiles each module with the larger of 128 and the state's size.
#define MPPI_MAX_STATE_BYTES 128
#endif
#ifndef MPPI_MAX_CONTROL_DIM
// Control dimension limit (shaders/mppi_core.h:33).
#define MPPI_MAX_CONTROL_DIM 16
#endif

// ---------------------------------------------------------------------------
// Callable ABI (shaders/mppi_core.h:11-26).  A plugin defines __device__
// functions with these shapes; the names are chosen in ModelPluginSpec.
//   dynamics      : in-place state update; rng_counter / rng_seed let a
//                   stochastic model draw its own Philox numbers.
//   stage cost    : running cost on (post-dynamics state, clamped control).
//   terminal cost : cost on the final state.
// The state pointer may be declared as uint8_t* (as in the reference) or as
// float* / a struct pointer: the library casts to the declared type.
// ---------------------------------------------------------------------------
typedef void (*MppiDynamicsFn)(uint8_t* state, const float* control,
                               const uint8_t* model_params, uint2 rng_counter,
                               uint32_t rng_seed);
typedef float (*MppiStageCostFn)(const uint8_t* state, const float* control,
                                 const uint8_t* model_params,
                                 const uint8_t* cost_params);
typedef float (*MppiTerminalCostFn)(const uint8_t* state,
                                    const uint8_t* model_params,
                                    const uint8_t* cost_params);

// Default costs used when a cost callable is not named
// (shaders/mppi_rollout.metal:11-28): both return zero.
__device__ __forceinline__ float mppi_default_stage_cost(const uint8_t*, const float*,
                                                         const uint8_t*, const uint8_t*) {
  return 0.0f;
}
__device__ __forceinline__ float mppi_default_terminal_cost(const uint8_t*, const uint8_t*,
                                                            const uint8_t*) {
  return 0.0f;
}

// ---------------------------------------------------------------------------
// Parameter-layout declaration (the ParamLayout contract of the reference's
// include/mppi_metal/mppi_types.hpp:88-94, whose README promises that
// initialize fails when the declared layout does not match the binding).
// A plugin may state the layout of the blobs its callables read:
//   MPPI_PARAM_LAYOUT(model_bytes, model_align, cost_bytes, cost_align, "schema")
//   MPPI_PARAM_LAYOUT_OF(ModelParamsT, CostParamsT, "schema")
// and the module then compiles only if the driver's ParamLayout agrees:
// equal blob sizes, an alignment that is 1 (unspecified) or a multiple of the
// declared one, and a schema_hash that is empty or equal to the declared
// string.  A plugin without the declaration is bound as the reference binds
// it (sizes checked against the blobs only).
// ---------------------------------------------------------------------------
template <int>
struct mppi_declared_param_layout {
  static constexpr bool declared = false;
  static constexpr unsigned long long model_size = 0, model_align = 1;
  static constexpr unsigned long long cost_size = 0, cost_align = 1;
  static constexpr const char* schema = "";
};
#define MPPI_PARAM_LAYOUT(MODEL_BYTES, MODEL_ALIGN, COST_BYTES, COST_ALIGN, SCHEMA) \
  template <>                                                                      \
  struct mppi_declared_param_layout<0> {                                           \
    static constexpr bool declared = true;                                         \
    static constexpr unsigned long long model_size = (MODEL_BYTES);                \
    static constexpr unsigned long long model_align = (MODEL_ALIGN);               \
    static constexpr unsigned long long cost_size = (COST_BYTES);                  \
    static constexpr unsigned long long cost_align = (COST_ALIGN);                 \
    static constexpr const char* schema = SCHEMA;                                  \
  };
#define MPPI_PARAM_LAYOUT_OF(MODEL_T, COST_T, SCHEMA) \
  MPPI_PARAM_LAYOUT(sizeof(MODEL_T), alignof(MODEL_T), sizeof(COST_T), alignof(COST_T), SCHEMA)

// ---------------------------------------------------------------------------
// Optional split stage cost (no counterpart in the reference).  A plugin
// whose stage cost is a sum of independent terms may declare
//   MPPI_STAGE_COST_SPLIT(stage_fn, part_fn, PARTS)
// with part_fn(state, control, model_params, cost_params, int part) returning
// part `part` of stage_fn's value (the parts sum to it).  For launches with
// few CTAs (latency-bound: each sample's serial chain sets the time), the
// library then runs a cooperative rollout form: PARTS lanes per sample all
// step the dynamics and each evaluates one part, so the chain per step
// carries 1/PARTS of the cost terms.
// ---------------------------------------------------------------------------
template <auto F>
struct mppi_stage_cost_split {
  static constexpr int parts = 0;
  template <class S>
  __device__ static float part(S, const float*, const uint8_t*, const uint8_t*, int) {
    return 0.0f;
  }
};
#define MPPI_STAGE_COST_SPLIT(STAGE_FN, PART_FN, PARTS)                               \
  template <>                                                                        \
  struct mppi_stage_cost_split<&STAGE_FN> {                                          \
    static constexpr int parts = (PARTS);                                            \
    template <class S>                                                               \
    __device__ static float part(S s, const float* u, const uint8_t* mp,             \
                                 const uint8_t* cp, int j) {                         \
      return PART_FN(s, u, mp, cp, j);                                               \
    }                                                                                \
  };

// First-parameter type of a plain function, so the library can hand a
// plugin its state in whatever pointer type the plugin declared.
template <class F>
struct mppi_first_arg;
template <class R, class A0, class... As>
struct mppi_first_arg<R (*)(A0, As...)> {
  typedef A0 type;
};

// ---------------------------------------------------------------------------
// Philox-2x32-10 (shaders/philox.h:19-36).
//   round: (c0, c1) -> (hi(c0 * M) ^ key ^ c1, lo(c0 * M)),  M = 0xD256D193
//   key  : += 0x9E3779B9 after each of the 10 rounds
// ---------------------------------------------------------------------------
#define MPPI_PHILOX_M 0xD256D193u
#define MPPI_PHILOX_W 0x9E3779B9u

__device__ __forceinline__ uint2 mppi_philox2x32_10(uint2 ctr, uint32_t key) {
  uint32_t c0 = ctr.x, c1 = ctr.y;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const uint32_t hi = __umulhi(c0, MPPI_PHILOX_M);
    const uint32_t lo = c0 * MPPI_PHILOX_M;
    c0 = hi ^ key ^ c1;
    c1 = lo;
    key += MPPI_PHILOX_W;
  }
  return make_uint2(c0, c1);
}

// (float(x) + 0.5f) * 2^-32 (shaders/philox.h:39-41): two correctly rounded
// float operations, so the result is bit-identical to the reference's.
__device__ __forceinline__ float mppi_uint_to_01(uint32_t x) {
  const float f = __fadd_rn(__uint2float_rn(x), 0.5f);
  return __fmul_rn(f, 2.3283064365386962890625e-10f);
}

// Square root by the SM's approximate square-root instruction (PTX
// sqrt.approx.ftz.f32, relative error of order 2^-23), exact zero at zero.
// Subnormal inputs (below 2^-126) flush to zero and give 0: that keeps it a
// single instruction -- the form without .ftz adds a rescaling path for
// subnormals, which measured about four more instructions per call.  Used
// for the Box-Muller radius and by plugins for cost terms.
__device__ __forceinline__ float mppi_sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// ---------------------------------------------------------------------------
// The library's own sine / cosine.  Both reduce the argument exactly (or with
// an error far below float rounding) to a quarter turn around zero and
// evaluate near-minimax polynomials there.  The coefficients were fitted for
// this library (csrc/device/derive_poly.py: Lawson's iteratively reweighted
// least squares, then rounded to float); that script also reports the error
// of the float32 FMA evaluation below against float64 sin / cos.
// Quadrant q (x = q * pi/2 + r):  q%4 = 0: ( s,  c)  1: ( c, -s)
//                                        2: (-s, -c)  3: (-c,  s)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mppi_quadrant(uint32_t q, float s, float c, float* so,
                                              float* co) {
  const bool swap = (q & 1u) != 0u;
  const float a = swap ? c : s, b = swap ? s : c;
  *so = __uint_as_float(__float_as_uint(a) ^ ((q & 2u) << 30));
  *co = __uint_as_float(__float_as_uint(b) ^ (((q + 1u) & 2u) << 30));
}

// (sin(pi/2 v), cos(pi/2 v)) for |v| < 2^22: q = rint(v) by the 1.5 * 2^23
// rounding constant, and f = v - q is exact (|f| <= 1/2, Sterbenz), so the
// only errors are the polynomials' (at most 8.3e-8 for sin and 5.8e-8 for cos,
// absolute).
__device__ __forceinline__ void mppi_sincos_quarter(float v, float* so, float* co) {
  const float t = __fadd_rn(v, 0x1.8p23f);
  const float q = __fsub_rn(t, 0x1.8p23f);
  const float f = __fsub_rn(v, q);
  const float z = __fmul_rn(f, f);
  float ps = fmaf(-0x1.2d930ep-8f, z, 0x1.465e92p-4f);
  ps = fmaf(ps, z, -0x1.4abbbap-1f);
  ps = fmaf(ps, z, 0x1.921fb6p+0f);
  float pc = fmaf(0x1.d9f7c8p-11f, z, -0x1.55c664p-6f);
  pc = fmaf(pc, z, 0x1.03c1dep-2f);
  pc = fmaf(pc, z, -0x1.3bd3ccp+0f);
  mppi_quadrant(__float_as_uint(t), __fmul_rn(f, ps), fmaf(pc, z, 1.0f), so, co);
}

// sin and cos of x (radians), for plugins.  Cody and Waite's reduction by
// pi/2 (W. J. Cody, W. Waite, "Software Manual for the Elementary Functions",
// 1980) with FMAs and pi/2 split into two floats: |x| < 65536 keeps the
// reduction error below 1.2e-10; beyond that the call falls back to CUDA's
// sincosf.  Error at most 4.4e-8 (sin) and 5.3e-8 (cos) absolute on the
// reduced argument.
__device__ __forceinline__ void mppi_sincosf(float x, float* so, float* co) {
  if (!(fabsf(x) < 65536.0f)) {
    sincosf(x, so, co);
    return;
  }
  const float t = fmaf(x, 0x1.45f306p-1f, 0x1.8p23f);  // x * 2/pi + 1.5 * 2^23
  const float q = __fsub_rn(t, 0x1.8p23f);
  float r = fmaf(-q, 0x1.921fb6p+0f, x);
  r = fmaf(-q, -0x1.777a5cp-25f, r);
  const float z = __fmul_rn(r, r);
  float ps = fmaf(-0x1.9943f2p-13f, z, 0x1.11073cp-7f);
  ps = fmaf(ps, z, -0x1.555546p-3f);
  float pc = fmaf(0x1.99343ap-16f, z, -0x1.6c087ep-10f);
  pc = fmaf(pc, z, 0x1.55553ep-5f);
  pc = fmaf(pc, z, -0.5f);
  mppi_quadrant(__float_as_uint(t), fmaf(ps, __fmul_rn(r, z), r), fmaf(pc, z, 1.0f), so, co);
}

// ln x for normal x > 0 (the Box-Muller argument u1 lies in [2^-33, 1]): the
// exponent is split off around 2/3, x = 2^e (1 + f) with f in [-1/3, 1/3)
// exact (Sterbenz), and ln(1 + f) = f + f^2 P(f) with a degree-7 polynomial
// fitted for this library (csrc/device/derive_poly.py); e ln 2 is added in two
// parts (the first exact).  Relative error at most 8.7e-8 on the Box-Muller
// arguments (float32 evaluation against float64).  Not for zero, negative,
// subnormal, infinite or NaN arguments.
__device__ __forceinline__ float mppi_log(float x) {
  const uint32_t i = __float_as_uint(x);
  const int32_t e = (int32_t)(i - 0x3f2aaaabu) >> 23;
  const float f = __fsub_rn(__uint_as_float(i - ((uint32_t)e << 23)), 1.0f);
  float p = fmaf(0x1.1f421ap-3f, f, -0x1.3b27cap-3f);
  p = fmaf(p, f, 0x1.1ea26ap-3f);
  p = fmaf(p, f, -0x1.5032fep-3f);
  p = fmaf(p, f, 0x1.99d426p-3f);
  p = fmaf(p, f, -0x1.00147ep-2f);
  p = fmaf(p, f, 0x1.5554fap-2f);
  p = fmaf(p, f, -0x1.ffffd6p-2f);
  const float r = fmaf(p, __fmul_rn(f, f), f);
  const float ef = (float)e;
  return fmaf(ef, 0x1.62e4p-1f, fmaf(ef, 0x1.7f7d1cp-20f, r));
}

// Box-Muller (shaders/philox.h:44-50): r = sqrt(-2 ln u1), theta = 2 pi u2.
// The angle is taken as a quarter-turn count, 4 u2 = (x2 + 0.5) * 2^-30 --
// exactly 4 times the reference's u2 -- so 2 pi u2 is never rounded to a
// float; the library's logarithm gives ln u1 and the SM's square root the
// radius (relative error of order 2^-23).
__device__ __forceinline__ float2 mppi_box_muller(uint2 w) {
  const float u1 = mppi_uint_to_01(w.x);
  const float v = __fmul_rn(__fadd_rn(__uint2float_rn(w.y), 0.5f), 0x1p-30f);
  const float r = mppi_sqrt_approx(-2.0f * mppi_log(u1));
  float s, c;
  mppi_sincos_quarter(v, &s, &c);
  return make_float2(r * c, r * s);
}

// Half-precision noise mode (DriverConfig::NumericMode kFp16 / kMixed): the
// shaped noise is rounded once to IEEE binary16 (round to nearest even) and
// that rounded value is used everywhere -- rollout and weighted update alike.
__device__ __forceinline__ uint16_t mppi_f32_to_f16(float x) {
  uint16_t h;
  asm("cvt.rn.f16.f32 %0, %1;" : "=h"(h) : "f"(x));
  return h;
}
__device__ __forceinline__ float mppi_f16_to_f32(uint16_t h) {
  float f;
  asm("cvt.f32.f16 %0, %1;" : "=f"(f) : "h"(h));
  return f;
}


// Box-Muller with the SM's approximate log2 / sqrt / sin / cos (relative
// errors of order 2^-21), for the half-precision noise mode whose output is
// rounded to 11 significant bits anyway.  The angle is taken as
// 2 pi (u2 - 1/2), inside (-pi, pi) where the approximate sine / cosine are
// accurate, and sin / cos(t + pi) = -sin / cos(t) restores the reference's
// angle 2 pi u2.
__device__ __forceinline__ float2 mppi_box_muller_fast(uint2 w) {
  const float u1 = mppi_uint_to_01(w.x);
  const float u2 = mppi_uint_to_01(w.y);
  const float r = mppi_sqrt_approx(-2.0f * __logf(u1));
  float s, c;
  __sincosf(6.28318530717958647692f * (u2 - 0.5f), &s, &c);
  return make_float2(-r * c, -r * s);
}

// The same from one 32-bit Philox word split into two 16-bit uniforms,
// u = (h + 1/2) 2^-16 (lower half u1, upper half u2), for the half-precision
// noise mode of models with three or more controls: 16 bits of uniform
// suffice for a normal rounded to 11 significant bits, so one Philox call
// gives four normals instead of two (its tails end at 4.9 sigma, where
// u1 = 2^-17).
__device__ __forceinline__ float2 mppi_box_muller_fast16(uint32_t w) {
  const float u1 = __fmul_rn(__fadd_rn(__uint2float_rn(w & 0xffffu), 0.5f), 0x1p-16f);
  const float u2 = __fmul_rn(__fadd_rn(__uint2float_rn(w >> 16), 0.5f), 0x1p-16f);
  const float r = mppi_sqrt_approx(-2.0f * __logf(u1));
  float s, c;
  __sincosf(6.28318530717958647692f * (u2 - 0.5f), &s, &c);
  return make_float2(-r * c, -r * s);
}

// Reference-compatible spellings for plugins ported from MSL
// (examples/wez_environment_batch/wez_environment.metal:166-173 draws with
// philox2x32_10 / uint_to_01 inside its dynamics).
__device__ __forceinline__ uint2 philox2x32_10(uint2 ctr, uint32_t key) {
  return mppi_philox2x32_10(ctr, key);
}
__device__ __forceinline__ float uint_to_01(uint32_t x) { return mppi_uint_to_01(x); }
__device__ __forceinline__ float2 box_muller(uint2 w) { return mppi_box_muller(w); }

// Counter layout of the reference (shaders/mppi_rollout.metal:66-90):
//   noise pair  (step, k*H*P + t*P + d/2)          P = ceil(m/2)
//   dynamics    (step, k*H*P + t + 0x80000000)
//   propagate   (step, 0x80000000)                  (mppi_reduce.metal:212)
// All arithmetic wraps modulo 2^32 exactly as the reference's uint math.
__device__ __forceinline__ uint32_t mppi_noise_ctr(uint32_t k, uint32_t H, uint32_t P,
                                                   uint32_t t, uint32_t pair) {
  return k * H * P + t * P + pair;
}
__device__ __forceinline__ uint32_t mppi_dyn_ctr(uint32_t k, uint32_t H, uint32_t P,
                                                 uint32_t t) {
  return k * H * P + t + 0x80000000u;
}
