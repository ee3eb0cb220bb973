// mppi_kernels.cuh — the MPPI hot path for sm_100a, compiled by NVRTC once per
// driver together with the user's model plugin (csrc/nvrtc_module.cpp), so
// the dynamics / cost callables inline into the rollout and the state stays
// in registers.
//
// Compile-time configuration (NVRTC -D options set by the backend):
//   MPPI_STATE_DIM, MPPI_CONTROL_DIM        problem dimensions
//   MPPI_COV_FULL                           0: sigma = per-dim std-dev
//                                           1: sigma = Cholesky factor L
//   MPPI_CONTROL_COST                       1: add lambda * u_nom^T Sigma^-1 eps
//   MPPI_NOISE_HALF                         1: noise drawn with approximate
//                                           transcendentals (four 16-bit
//                                           uniforms per Philox call for
//                                           m >= 3), rounded to FP16, staged
//                                           in FP16 (kFp16 / kMixed)
//   MPPI_DYNAMICS_FN / _STAGE_COST_FN / _TERMINAL_COST_FN   callable names
//   MPPI_MP_BYTES / MPPI_CP_BYTES           ParamLayout blob sizes
//   MPPI_PROPOSAL                           1: a share of the samples draws
//                                           around a learned proposal
//                                           (MppiRolloutArgs::prop_out)
//   MPPI_FEATURES_FN                        the plugin's proposal-feature
//                                           callable (mppi_features kernel)
//
// Kernels (extern "C" names are looked up by the backend):
//   mppi_rollout_b{64,128,256}  fused rollout + per-CTA softmax partials +
//                               weighted-noise partial sums
//   mppi_rollout_fused_b{...}   the same + each agent's combine in its last CTA
//   mppi_rollout_work[_fused]_b128  the same for uneven batches (work items)
//   mppi_rollout_ws[_fused]_b128    warp-specialised form (noise drawn by a
//                               second set of warps one chunk ahead)
//   mppi_combine                per-agent combine -> u_out, diagnostics,
//                               optional propagate & shift (closed loop)
//   mppi_weights                normalised weights (inspection only)
//   mppi_noise                  shaped noise of a sample range (inspection)
//   mppi_features               proposal features of state rows (only with
//                               MPPI_FEATURES_FN)
//
// Reference semantics followed (MarshallVielmetti/mppi_metal):
//   rollout          shaders/mppi_rollout.metal:36-96 and :103-170
//   weights          shaders/mppi_reduce.metal:14-121  (w = exp(-(c-min)/l)/sum)
//   update           shaders/mppi_reduce.metal:130-168 (unclamped noise, Q6)
//   propagate/shift  shaders/mppi_reduce.metal:175-231 and :413-488
// The reference runs these as four passes and regenerates every noise value
// in a serial k-loop of the update pass.  Here the rollout CTA keeps its
// samples' noise in shared memory, and once its costs are known it reduces
// sum_k e_k * eps_k for its samples with e_k = exp(-(c_k - m_b) / lambda)
// taken against the CTA's own minimum m_b.  The combine kernel rescales the
// CTA partials to the global minimum M (e_k * exp(-(m_b - M) / lambda)),
// which gives the reference's weights exactly in exact arithmetic.
#pragma once

#include "mppi_launch.h"
#include "mppi_gelu.cuh"

#ifndef MPPI_STATE_DIM
#error "MPPI_STATE_DIM must be defined"
#endif
#ifndef MPPI_CONTROL_DIM
#error "MPPI_CONTROL_DIM must be defined"
#endif
#ifndef MPPI_COV_FULL
#define MPPI_COV_FULL 0
#endif
#ifndef MPPI_CONTROL_COST
#define MPPI_CONTROL_COST 0
#endif
#ifndef MPPI_NOISE_HALF
#define MPPI_NOISE_HALF 0
#endif
#ifndef MPPI_PROPOSAL
#define MPPI_PROPOSAL 0
#endif
#ifndef MPPI_MP_BYTES
#define MPPI_MP_BYTES 0
#endif
// Features per row of the proposal network's input.
#define MPPI_MAX_FEATURES 32
#ifndef MPPI_CP_BYTES
#define MPPI_CP_BYTES 0
#endif
// ParamLayout alignments and schema_hash (checked against a plugin's
// MPPI_PARAM_LAYOUT declaration)
#ifndef MPPI_MP_ALIGN
#define MPPI_MP_ALIGN 1
#endif
#ifndef MPPI_CP_ALIGN
#define MPPI_CP_ALIGN 1
#endif
#ifndef MPPI_SCHEMA_HASH
#define MPPI_SCHEMA_HASH ""
#endif
#ifndef MPPI_STAGE_COST_FN
#define MPPI_STAGE_COST_FN mppi_default_stage_cost
#endif
#ifndef MPPI_TERMINAL_COST_FN
#define MPPI_TERMINAL_COST_FN mppi_default_terminal_cost
#endif

// Parameter blobs up to this size are copied into shared memory once per CTA
// and the callables read them from there (uniform broadcast loads).
#define MPPI_PARAM_SMEM_MAX 8192
#define MPPI_MP_SMEM (MPPI_MP_BYTES > 0 && MPPI_MP_BYTES <= MPPI_PARAM_SMEM_MAX)
#define MPPI_CP_SMEM (MPPI_CP_BYTES > 0 && MPPI_CP_BYTES <= MPPI_PARAM_SMEM_MAX)

namespace mppi {

constexpr int kN = MPPI_STATE_DIM;
constexpr int kM = MPPI_CONTROL_DIM;
constexpr int kP = (kM + 1) / 2;        // Philox pairs per time step
constexpr int kNPad = (kN + 3) / 4 * 4;  // state buffer, 16-byte multiple
constexpr int kSig = MPPI_COV_FULL ? kM * kM : kM;
constexpr unsigned kFull = 0xffffffffu;

static_assert(kN >= 1 && kN * 4 <= MPPI_MAX_STATE_BYTES, "state_dim out of range");
static_assert(kM >= 1 && kM <= MPPI_MAX_CONTROL_DIM, "control_dim out of range");

// ---- ParamLayout against the plugin's declared layout (MPPI_PARAM_LAYOUT) ----
// The messages carry a marker the host looks for in the compile log.
__host__ __device__ constexpr bool str_eq(const char* a, const char* b) {
  while (*a != '\0' && *a == *b) {
    ++a;
    ++b;
  }
  return *a == *b;
}
typedef mppi_declared_param_layout<0> DeclaredLayout;
static_assert(!DeclaredLayout::declared || DeclaredLayout::model_size == MPPI_MP_BYTES,
              "MPPI_PARAM_LAYOUT_MISMATCH: ParamLayout::model_params_size differs from the "
              "model parameter size the plugin declares");
static_assert(!DeclaredLayout::declared || DeclaredLayout::cost_size == MPPI_CP_BYTES,
              "MPPI_PARAM_LAYOUT_MISMATCH: ParamLayout::cost_params_size differs from the "
              "cost parameter size the plugin declares");
static_assert(!DeclaredLayout::declared || MPPI_MP_ALIGN == 1 ||
                  MPPI_MP_ALIGN % DeclaredLayout::model_align == 0,
              "MPPI_PARAM_LAYOUT_MISMATCH: ParamLayout::model_params_alignment is not a multiple "
              "of the model parameter alignment the plugin declares");
static_assert(!DeclaredLayout::declared || MPPI_CP_ALIGN == 1 ||
                  MPPI_CP_ALIGN % DeclaredLayout::cost_align == 0,
              "MPPI_PARAM_LAYOUT_MISMATCH: ParamLayout::cost_params_alignment is not a multiple "
              "of the cost parameter alignment the plugin declares");
static_assert(!DeclaredLayout::declared || str_eq(MPPI_SCHEMA_HASH, "") ||
                  str_eq(MPPI_SCHEMA_HASH, DeclaredLayout::schema),
              "MPPI_PARAM_LAYOUT_MISMATCH: ParamLayout::schema_hash differs from the schema "
              "the plugin declares");

typedef typename mppi_first_arg<decltype(&MPPI_DYNAMICS_FN)>::type DynStateT;
typedef typename mppi_first_arg<decltype(&MPPI_STAGE_COST_FN)>::type StageStateT;
typedef typename mppi_first_arg<decltype(&MPPI_TERMINAL_COST_FN)>::type TermStateT;

__device__ __forceinline__ float pos_inf() { return __int_as_float(0x7f800000); }

// Programmatic dependent launch (launches with the programmatic stream
// serialisation attribute): a CTA lets the next kernel in the stream be
// scheduled as soon as it has started, and the next kernel's CTAs run their
// loop-constant prologue before they wait for this grid to complete and its
// memory to be visible.  Both are no-ops in launches without the attribute.
__device__ __forceinline__ void mppi_allow_dependent_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void mppi_grid_dependency_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Element type of the shared-memory noise staging buffer.
#if MPPI_NOISE_HALF
typedef uint16_t stage_t;
__device__ __forceinline__ stage_t to_stage(float x) { return mppi_f32_to_f16(x); }
__device__ __forceinline__ float from_stage(stage_t h) { return mppi_f16_to_f32(h); }
#else
typedef float stage_t;
__device__ __forceinline__ stage_t to_stage(float x) { return x; }
__device__ __forceinline__ float from_stage(stage_t x) { return x; }
#endif

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Sample costs are accumulated as an unevaluated pair hi + lo of floats:
// Knuth's TwoSum gives the exact rounding error of every addition to hi,
// and lo collects those errors.  With lambda = 1 and costs of order 1e3-1e4
// the softmax turns the plain float sum's rounding (an ulp of the running
// total per step, about 5e-4 at 8e3) into weight errors of the same size;
// the pair keeps the accumulated total to the rounding of the cost terms
// themselves.  Additions only (no multiply to contract into an FMA).
__device__ __forceinline__ void acc_cost(float& hi, float& lo, float x) {
  const float s = hi + x;
  const float bp = s - hi;
  const float err = (hi - (s - bp)) + (x - bp);
  hi = s;
  lo += err;
}

// A load through L2 that the compiler keeps where it is written (volatile
// asm): the combine issues its reads of other CTAs' records ahead of the
// statistics that wait on them, so they overlap instead of following.
__device__ __forceinline__ float ld_early(const float* p) {
  float v;
  asm volatile("ld.global.cg.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

// The pair as one double (exact: |lo| is far below hi's last bit times 2^29).
__device__ __forceinline__ double cost_pair(float hi, float lo) {
  return (double)hi + (double)lo;
}
__device__ __forceinline__ float pair_hi(double v) { return (float)v; }
__device__ __forceinline__ float pair_lo(double v) { return (float)(v - (double)(float)v); }

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
  // Metal clamp(x, lo, hi) = min(max(x, lo), hi)
  return fminf(fmaxf(v, lo), hi);
}

// Standard normals n[0..m) and shaped noise eps[0..m) of sample k at time t.
// Pair p of step t uses counter (step, k*H*P + t*P + p); its first normal is
// dim 2p, its second dim 2p+1 (dropped for odd m).
// Half-precision noise with three or more controls: one Philox call per
// four normals (mppi_box_muller_fast16), call q of step t at counter
// (step, k*H*Q + t*Q + q), Q = ceil(m/4); its word x gives dims 4q, 4q+1,
// word y dims 4q+2, 4q+3.
constexpr bool kNoise16 = MPPI_NOISE_HALF && kM >= 3;
constexpr int kQ = (kM + 3) / 4;

__device__ __forceinline__ void sample_noise(uint32_t step, uint32_t key, uint32_t k,
                                             uint32_t H, uint32_t t, const float (&sig)[kSig],
                                             float (&n)[2 * kP], float (&eps)[kM]) {
  if constexpr (kNoise16) {
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const uint2 w = mppi_philox2x32_10(make_uint2(step, mppi_noise_ctr(k, H, kQ, t, q)), key);
      const float2 g0 = mppi_box_muller_fast16(w.x);
      n[4 * q] = g0.x;
      if (4 * q + 1 < kM) n[4 * q + 1] = g0.y;
      if (4 * q + 2 < kM) {
        const float2 g1 = mppi_box_muller_fast16(w.y);
        n[4 * q + 2] = g1.x;
        if (4 * q + 3 < kM) n[4 * q + 3] = g1.y;
      }
    }
  }
#pragma unroll
  for (int p = 0; p < (kNoise16 ? 0 : kP); ++p) {
    const uint2 w = mppi_philox2x32_10(make_uint2(step, mppi_noise_ctr(k, H, kP, t, p)), key);
#if MPPI_NOISE_HALF
    const float2 g = mppi_box_muller_fast(w);
#else
    const float2 g = mppi_box_muller(w);
#endif
    n[2 * p] = g.x;
    n[2 * p + 1] = g.y;
  }
#if MPPI_COV_FULL
#pragma unroll
  for (int d = 0; d < kM; ++d) {
    float e = 0.0f;
#pragma unroll
    for (int j = 0; j <= d; ++j) e = fmaf(sig[d * kM + j], n[j], e);
    eps[d] = e;
  }
#else
#pragma unroll
  for (int d = 0; d < kM; ++d) eps[d] = n[d] * sig[d];
#endif
#if MPPI_NOISE_HALF
#pragma unroll
  for (int d = 0; d < kM; ++d) eps[d] = from_stage(to_stage(eps[d]));
#endif
}

__device__ __forceinline__ void load_sigma(const float* g, float (&sig)[kSig]) {
#pragma unroll
  for (int i = 0; i < kSig; ++i) sig[i] = g[i];
}

// Copies `bytes` (a multiple of 4 after padding) from global to shared memory.
__device__ __forceinline__ void copy_words(uint32_t* dst, const uint8_t* src, int bytes) {
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  for (int i = threadIdx.x; i < (bytes + 3) / 4; i += blockDim.x) dst[i] = s[i];
}

// Proposal samples replace the plain draw eps = sigma n by
// (mu - u_nom) + exp(s) n on the same standard normals n (rounded like the
// plain draw in the FP16 modes).  The branch is uniform over a warp (the
// proposal samples are a prefix of k).
#if MPPI_PROPOSAL
#define MPPI_PROPOSAL_EPS()                                                       \
  do {                                                                            \
    if (k < pcount) {                                                             \
      _Pragma("unroll") for (int d_ = 0; d_ < kM; ++d_) eps[d_] =                 \
          from_stage(to_stage(fmaf(ps_s[d_], n[d_], sh_s[t * kM + d_])));          \
    }                                                                             \
  } while (0)
#else
#define MPPI_PROPOSAL_EPS() \
  do {                      \
  } while (0)
#endif

// --------------------------------------------------------------------------
// Fused rollout of one work item: CTA `blk` of agent `agent` (K samples,
// horizon H, nominal at un_g, partial record at part).  One thread per
// sample.  Dynamic shared memory: u_nom[H*m] | staging[stage_rows][BLOCK] |
// e[BLOCK] (sized for the launch's largest horizon).
//
// WS (warp-specialised form, 2 * BLOCK threads, whole horizon staged): the
// second BLOCK threads draw the noise of sample column tid - BLOCK a chunk of
// kWsChunk steps ahead while the first BLOCK threads run the state
// recurrence of the previous chunk; one CTA barrier hands each chunk over.
// Each sample's chain then carries only the dynamics and costs -- for launches
// whose few CTAs leave SMs idle (latency-bound), not for full ones.  The
// extra warps add exact zeros (and +inf to the minimum) to the CTA
// statistics, so the results are the same bits as the plain form.
// --------------------------------------------------------------------------
//
// LANES > 1 (cooperative form; the plugin's stage cost split into LANES parts
// by MPPI_STAGE_COST_SPLIT, BLOCK * LANES threads): the LANES consecutive
// threads of a sample share its staged noise (each draws every LANES-th
// step), all step the dynamics, and each accumulates one part of the stage
// cost (part 0 also the control and terminal costs); the parts are summed as
// doubles by a butterfly of shuffles at the end, ((p0 + p1) + (p2 + p3)) for
// four.  A sample's cost then sums its terms in another order than the other
// forms, so its bits differ from theirs in the last places.
// --------------------------------------------------------------------------
constexpr uint32_t kWsChunk = 4;

typedef mppi_stage_cost_split<&MPPI_STAGE_COST_FN> StageSplit;
// Lanes per sample of the cooperative form (0: the plugin declares no split).
constexpr int kCoopLanes = StageSplit::parts;
static_assert(kCoopLanes == 0 || kCoopLanes == 2 || kCoopLanes == 4,
              "MPPI_STAGE_COST_SPLIT: the part count must be 2 or 4");

template <int BLOCK, bool WS = false, int LANES = 1, bool EARLY = false>
__device__ __forceinline__ void rollout_item(const MppiRolloutArgs& a, uint32_t agent,
                                             uint32_t blk, uint32_t K, uint32_t H,
                                             const float* un_g, float* part) {
  static_assert(!(WS && LANES > 1), "the cooperative form is not warp-specialised");
  constexpr int NT = WS ? 2 * BLOCK : BLOCK * LANES;  // threads of the CTA
  constexpr int NW = NT / 32;
  constexpr int PER_LANE = BLOCK / 32;
  static_assert(BLOCK % 32 == 0, "sample columns come in warps");
  extern __shared__ __align__(16) float dsm[];
  __shared__ double wmin_s[NW];    // per-warp minimum costs
  __shared__ float wsum_s[3 * NW];  // per-warp sums of e, e^2 and the costs
#if MPPI_MP_SMEM
  __shared__ __align__(16) uint32_t mp_s[(MPPI_MP_BYTES + 3) / 4];
#endif
#if MPPI_CP_SMEM
  __shared__ __align__(16) uint32_t cp_s[(MPPI_CP_BYTES + 3) / 4];
#endif

  const uint32_t tid = threadIdx.x;
  const uint32_t lane = tid & 31, warp = tid >> 5;
  const bool producer = WS && tid >= (uint32_t)BLOCK;  // noise-drawing warp (WS form)
  // this thread's sample column, and its part of the sample (cooperative form)
  const uint32_t col = WS ? tid % BLOCK : tid / LANES;
  const uint32_t sub = tid % LANES;
  const uint32_t HM = H * kM;
  const uint32_t k = blk * BLOCK + col;
  const bool active = k < K;
  const uint32_t step = *a.step_base + a.step_local;
  const uint32_t key = a.seed + agent;
  const bool staged = a.stage_rows >= HM;

  const uint32_t HMp = (a.H * kM + 3) & ~3u;
  float* un_s = dsm;
#if MPPI_PROPOSAL
  float* sh_s = dsm + HMp;  // proposal mean shift mu - u_nom
  stage_t* stage_s = reinterpret_cast<stage_t*>(dsm + 2 * HMp);
#else
  stage_t* stage_s = reinterpret_cast<stage_t*>(dsm + HMp);
#endif
  float* e_s = reinterpret_cast<float*>(stage_s + (size_t)a.stage_rows * BLOCK);

  const uint8_t* mp_g = a.model_params + a.model_stride * agent;
  const uint8_t* cp_g = a.cost_params + a.cost_stride * agent;
#if MPPI_MP_SMEM
  copy_words(mp_s, mp_g, MPPI_MP_BYTES);
  const uint8_t* mp = reinterpret_cast<const uint8_t*>(mp_s);
#else
  const uint8_t* mp = mp_g;
#endif
#if MPPI_CP_SMEM
  copy_words(cp_s, cp_g, MPPI_CP_BYTES);
  const uint8_t* cp = reinterpret_cast<const uint8_t*>(cp_s);
#else
  const uint8_t* cp = cp_g;
#endif
  float sig[kSig], lo[kM], hi[kM];
  load_sigma(a.sigma + (size_t)a.sigma_stride * agent, sig);
#pragma unroll
  for (int d = 0; d < kM; ++d) {
    lo[d] = a.u_min[d];
    hi[d] = a.u_max[d];
  }
#if MPPI_CONTROL_COST
  float sinv[kSig];
  load_sigma(a.sigma_inv + (size_t)a.sigma_inv_stride * agent, sinv);
#endif
#if MPPI_PROPOSAL
  // samples k < pcount draw around the network's predicted sequence; the
  // shift and the scales live in shared memory, not in registers, so the
  // rollout's register budget stays the plain kernel's
  __shared__ float ps_s[kM];
  const uint32_t pcount = a.prop_out ? a.prop_count : 0u;
#else
  constexpr uint32_t pcount = 0;
#endif
  // Early noise: the noise depends on the step index, the sample and the
  // agent's sigma only -- nothing an earlier launch writes -- so without a
  // proposal the first chunk of it (the whole horizon when the staging
  // buffer holds it) is drawn before the wait for the previous launch.  A
  // step whose CTAs are resident early (a launch of few CTAs, programmatic
  // dependent launch) draws it while the previous step still runs, off the
  // critical path.  The values are the ones drawn after the wait would be.
  // Compiled in where EARLY is set (the cooperative entries and the
  // mppi_rollout_early_* entries, which the host launches with the whole
  // horizon staged), so the other kernels keep their register allocation.
  const bool early = EARLY && !WS && pcount == 0u;
  float J = 0.0f, Jlo = 0.0f;  // the sample's cost as the pair J + Jlo (acc_cost)
  __align__(16) float st[kNPad];
  const bool runs = active && !producer;  // this thread runs a sample's recurrence
#pragma unroll
  for (int d = kN; d < kNPad; ++d) st[d] = 0.0f;
  // The wait for the previous launch, then what it wrote: the nominal, the
  // proposal's output and (MPPI_LOAD_STATE, at each call site: no register
  // array captured by the lambda) the state.  Everything before it is
  // constant over a closed loop.  Ends with a CTA barrier (the nominal, the
  // proposal's shift and any noise rows drawn before it visible to all).
#define MPPI_LOAD_STATE()                                \
  if (runs) {                                            \
    const float* xg_ = a.x + (size_t)agent * kN;         \
    _Pragma("unroll") for (int d_ = 0; d_ < kN; ++d_) st[d_] = xg_[d_]; \
  }
  auto wait_and_load = [&]() {
    mppi_grid_dependency_wait();
    for (uint32_t i = tid; i < HM; i += NT) un_s[i] = un_g[i];
#if MPPI_PROPOSAL
    if (pcount) {
      const float* po = a.prop_out + (size_t)agent * a.prop_stride;
      for (uint32_t i = tid; i < HM; i += NT)
        sh_s[i] = i < a.prop_ls_offset ? po[i] - un_g[i] : 0.0f;
      if (tid < (uint32_t)kM)
        ps_s[tid] = expf(clampf(po[a.prop_ls_offset + tid], a.prop_ls_min, a.prop_ls_max));
    }
#endif
    __syncthreads();
  };
  // Noise of step t into this thread's staging column (row (t - row0) * m + d).
  auto draw = [&](uint32_t t, uint32_t row0) {
    float n[2 * kP], eps[kM];
    if (active) {
      sample_noise(step, key, k, H, t, sig, n, eps);
      MPPI_PROPOSAL_EPS();
    } else {
#pragma unroll
      for (int d = 0; d < kM; ++d) eps[d] = 0.0f;
    }
#pragma unroll
    for (int d = 0; d < kM; ++d)
      stage_s[(size_t)((t - row0) * kM + d) * BLOCK + col] = to_stage(eps[d]);
  };
  // One step of the recurrence on the staged noise.
  auto advance = [&](uint32_t t, uint32_t row0) {
    float eps[kM], u[kM];
#pragma unroll
    for (int d = 0; d < kM; ++d) {
      eps[d] = from_stage(stage_s[(size_t)((t - row0) * kM + d) * BLOCK + col]);
      u[d] = clampf(un_s[t * kM + d] + eps[d], lo[d], hi[d]);
    }
    // the step's cost terms are added together first, then into the
    // compensated sum once (the control cost lambda * u_nom^T Sigma^-1 eps
    // with the stage cost, or with part 0 of a split stage cost)
    float cterm = 0.0f;
#if MPPI_CONTROL_COST
    {
      float cc = 0.0f;
#if MPPI_COV_FULL
#pragma unroll
      for (int i = 0; i < kM; ++i) {
        float r = 0.0f;
#pragma unroll
        for (int j = 0; j < kM; ++j) r = fmaf(sinv[i * kM + j], eps[j], r);
        cc = fmaf(un_s[t * kM + i], r, cc);
      }
#else
#pragma unroll
      for (int i = 0; i < kM; ++i) cc = fmaf(un_s[t * kM + i], sinv[i] * eps[i], cc);
#endif
      cterm = (LANES == 1 || sub == 0) ? a.lambda * cc : 0.0f;
    }
#endif
    MPPI_DYNAMICS_FN(reinterpret_cast<DynStateT>(reinterpret_cast<void*>(st)), u, mp,
                     make_uint2(step, mppi_dyn_ctr(k, H, kP, t)), key);
    if constexpr (LANES > 1)
      acc_cost(J, Jlo,
               StageSplit::part(reinterpret_cast<StageStateT>(reinterpret_cast<void*>(st)), u, mp,
                                cp, (int)sub) +
                   cterm);
    else
      acc_cost(J, Jlo,
               MPPI_STAGE_COST_FN(reinterpret_cast<StageStateT>(reinterpret_cast<void*>(st)), u,
                                  mp, cp) +
                   cterm);
  };
  // ---- rollout: noise -> clamp -> dynamics -> stage cost; terminal cost ----
  // Time is processed in chunks of TC steps (the whole horizon when the
  // staging buffer holds it).  Phase A draws the chunk's noise into this
  // sample's staging column: Philox chains of different steps are
  // independent, so they overlap.  Phase B runs the state recurrence,
  // reading the noise back.  No thread touches another sample's column until
  // the weighted sums, so the phases need no CTA barrier of their own; the
  // lanes of a cooperative sample (one warp) share a column and meet at a
  // warp barrier between the phases.  The wait for the previous launch comes
  // first, or (early noise) after the first chunk's phase A.
  if (!early) {
    wait_and_load();
    MPPI_LOAD_STATE();
  }
  if constexpr (WS) {
    if (staged) {
      // producers draw the first chunk (early noise: the whole horizon) and
      // then stay one chunk ahead; the barrier after each chunk makes the
      // next chunk's rows visible to the recurrence warps
      const uint32_t first = early ? H : min(H, kWsChunk);
      if (producer) {
#pragma unroll 4
        for (uint32_t t = 0; t < first; ++t) draw(t, 0u);
      }
      if (early) {
        wait_and_load();
        MPPI_LOAD_STATE();
      } else {
        __syncthreads();
      }
      for (uint32_t c0 = 0; c0 < H; c0 += kWsChunk) {
        if (producer) {
          if (!early) {
            const uint32_t n0 = c0 + kWsChunk, n1 = min(H, n0 + kWsChunk);
#pragma unroll 4
            for (uint32_t t = n0; t < n1; ++t) draw(t, 0u);
          }
        } else if (runs) {
          // a whole chunk unrolled: the compiler can start step t + 1's
          // dynamics while step t's cost terms are still in flight
          if (c0 + kWsChunk <= H) {
#pragma unroll
            for (uint32_t i = 0; i < kWsChunk; ++i) advance(c0 + i, 0u);
          } else {
            for (uint32_t t = c0; t < H; ++t) advance(t, 0u);
          }
        }
        if (!early) __syncthreads();
      }
    } else {
      if (early) wait_and_load();
      J = __int_as_float(0x7fc00000);  // the host never runs this form chunked: NaN marks it
    }
  } else {
    const uint32_t TC = staged ? H : a.stage_rows / kM;
    if (early && H == 0u) wait_and_load();
    for (uint32_t t0 = 0; t0 < H; t0 += TC) {
      const uint32_t t1 = min(H, t0 + TC);
      const uint32_t row0 = staged ? 0u : t0;
      if constexpr (LANES > 1) {
        // a lane draws every LANES-th step
#pragma unroll 4
        for (uint32_t t = t0 + sub; t < t1; t += LANES) draw(t, row0);
      } else {
#pragma unroll 4
        for (uint32_t t = t0; t < t1; ++t) draw(t, row0);
      }
      if (early && t0 == 0u) {
        wait_and_load();  // its CTA barrier also orders the lanes' rows
        MPPI_LOAD_STATE();
      } else if constexpr (LANES > 1) {
        __syncwarp();
      }
      if (runs) {
        if constexpr (LANES > 1) {
          // two steps per pass: step t + 1's dynamics can start while step
          // t's cost terms are in flight
#pragma unroll 2
          for (uint32_t t = t0; t < t1; ++t) advance(t, row0);
        } else {
          for (uint32_t t = t0; t < t1; ++t) advance(t, row0);
        }
      }
      if constexpr (LANES > 1) __syncwarp();
    }
  }
#undef MPPI_LOAD_STATE
  double Jd = __longlong_as_double(0x7ff0000000000000ll);  // +inf: no sample here
  if constexpr (LANES > 1) {
    // part 0 carries the terminal cost; the parts meet in a butterfly
    if (runs && sub == 0)
      acc_cost(J, Jlo,
               MPPI_TERMINAL_COST_FN(reinterpret_cast<TermStateT>(reinterpret_cast<void*>(st)),
                                     mp, cp));
    double Jp = cost_pair(J, Jlo);
#pragma unroll
    for (int o = 1; o < LANES; o <<= 1) Jp += __shfl_xor_sync(kFull, Jp, o);
    if (runs) Jd = Jp;
  } else if (runs) {
    acc_cost(J, Jlo,
             MPPI_TERMINAL_COST_FN(reinterpret_cast<TermStateT>(reinterpret_cast<void*>(st)), mp,
                                   cp));
    Jd = cost_pair(J, Jlo);
  }
  // one thread per sample counts below (part 0 of a cooperative sample)
  const bool counts = runs && sub == 0;
  if (counts && a.costs) {  // inspection calls only; agent stride: the largest K
    a.costs[(size_t)agent * a.K + k] = pair_hi(Jd);
    a.costs_lo[(size_t)agent * a.K + k] = pair_lo(Jd);
  }
  if (!counts) Jd = __longlong_as_double(0x7ff0000000000000ll);

  // ---- CTA softmax statistics against the CTA minimum ----
  // The minimum and the differences c_k - m_b are taken on the cost pairs
  // (as doubles), so exp(-(c_k - m_b) / lambda) sees no rounding of c_k.
  // Two CTA barriers: per-warp minima, then the e_k and per-warp sums; the
  // warps' values combine in warp order (the same bits for any schedule).
  {
    const double wm = warp_min_d(Jd);
    if (lane == 0) wmin_s[warp] = wm;
  }
  __syncthreads();
  double bmin = wmin_s[0];
#pragma unroll
  for (int i = 1; i < NW; ++i) bmin = fmin(bmin, wmin_s[i]);
  const float e = counts ? expf(-(float)(Jd - bmin) / a.lambda) : 0.0f;
  if (!producer && sub == 0) e_s[col] = e;
  {
    const float s_e = warp_sum(e), s_e2 = warp_sum(e * e),
                s_c = warp_sum(counts ? pair_hi(Jd) : 0.0f);
    if (lane == 0) {
      wsum_s[3 * warp + 0] = s_e;
      wsum_s[3 * warp + 1] = s_e2;
      wsum_s[3 * warp + 2] = s_c;
    }
  }
  __syncthreads();
  if (tid == 0) {
    float s_e = wsum_s[0], s_e2 = wsum_s[1], s_c = wsum_s[2];
#pragma unroll
    for (int i = 1; i < NW; ++i) {
      s_e += wsum_s[3 * i + 0];
      s_e2 += wsum_s[3 * i + 1];
      s_c += wsum_s[3 * i + 2];
    }
    part[0] = pair_hi(bmin);
    part[1] = s_e;
    part[2] = s_e2;
    part[3] = s_c;
    part[4] = pair_lo(bmin);
  }
  float e_r[PER_LANE];
#pragma unroll
  for (int i = 0; i < PER_LANE; ++i) e_r[i] = e_s[lane + 32 * i];

  // ---- weighted noise sums V[j] = sum_k e_k eps_k[j] over this CTA ----
  const uint32_t R = staged ? HM : a.stage_rows;  // rows per chunk (multiple of m)
  for (uint32_t r0 = 0; r0 < HM; r0 += R) {
    const uint32_t rows = min(R, HM - r0);
    const stage_t* base = stage_s;
    if (!staged) {
      // regenerate this chunk's noise (same counters, same values)
      __syncthreads();
      const uint32_t t0 = r0 / kM, t1 = (r0 + rows) / kM;
      if (!producer)
        for (uint32_t t = t0 + sub; t < t1; t += LANES) draw(t, t0);
      __syncthreads();
    } else {
      base = stage_s + (size_t)r0 * BLOCK;
    }
    if constexpr (BLOCK == 32) {
      // 32 samples (the cooperative 32-sample CTA): one thread per row, over
      // the samples from a rotated start (row r from sample r mod 32), so a
      // warp's shared-memory reads hit 32 different banks
      for (uint32_t r = tid; r < rows; r += NT) {
        const stage_t* row = base + (size_t)r * BLOCK;
        float s = 0.0f;
#pragma unroll
        for (uint32_t i = 0; i < 32u; ++i) {
          const uint32_t c = (i + r) & 31u;
          s = fmaf(e_s[c], from_stage(row[c]), s);
        }
        part[MPPI_PARTIAL_HEAD + r0 + r] = s;
      }
      continue;
    }
    // four rows per pass, so their loads and shuffle trees overlap; each
    // row's sum is formed as in the one-row loop that finishes the chunk
    uint32_t r = warp;
    for (; r + 3 * NW < rows; r += 4 * NW) {
      float s[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const stage_t* row = base + (size_t)(r + q * NW) * BLOCK;
        s[q] = 0.0f;
#pragma unroll
        for (int i = 0; i < PER_LANE; ++i)
          s[q] = fmaf(e_r[i], from_stage(row[lane + 32 * i]), s[q]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) s[q] = warp_sum(s[q]);
      if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) part[MPPI_PARTIAL_HEAD + r0 + r + q * NW] = s[q];
      }
    }
    for (; r < rows; r += NW) {
      const stage_t* row = base + (size_t)r * BLOCK;
      float s = 0.0f;
#pragma unroll
      for (int i = 0; i < PER_LANE; ++i) s = fmaf(e_r[i], from_stage(row[lane + 32 * i]), s);
      s = warp_sum(s);
      if (lane == 0) part[MPPI_PARTIAL_HEAD + r0 + r] = s;
    }
  }
}

template <int CB, uint32_t PRE>
__device__ __forceinline__ void combine_agent(const MppiCombineArgs& a, uint32_t agent,
                                              float* dsm);

// The combine fused into the rollout launch (a.agent_done set): after its
// partial record, the CTA counts itself done for its agent, and the agent's
// last CTA (the one that brings the count to nblk) runs the agent's combine
// and resets the count.  The "last block" pattern, with no CTA waiting on
// another: the CTA barrier orders every thread's record stores before thread
// 0's count, an atomic add with release and acquire semantics at device
// scope, so the CTA that counts last sees every other CTA's record complete
// (and its barrier hands that on to its other threads).  One atomic replaces
// a device-scope fence on each side of a relaxed add.
__device__ __forceinline__ uint32_t atomic_add_acq_rel(uint32_t* p, uint32_t v) {
  uint32_t old;
  asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}

template <int BLOCK, uint32_t PRE = 32>
__device__ __forceinline__ void fused_combine_tail(const MppiRolloutArgs& a, uint32_t agent,
                                                   uint32_t nblk) {
  __shared__ uint32_t last_s;
  __syncthreads();  // this CTA's partial record complete, the staging memory free for reuse
  if (threadIdx.x == 0) last_s = atomic_add_acq_rel(a.agent_done + agent, 1u) + 1u == nblk;
  __syncthreads();
  if (!last_s) return;
  extern __shared__ __align__(16) float dsm_c[];
  combine_agent<BLOCK, PRE>(a.comb, agent, dsm_c);
  if (threadIdx.x == 0) a.agent_done[agent] = 0u;
}

// Uniform batch: grid (nblk, num_agents), every agent K samples, horizon H.
// FUSED: the kernel form with the combine tail (a separate entry point, so
// the plain form keeps its register allocation).
template <int BLOCK, bool FUSED, bool WS = false, int LANES = 1, bool EARLY = false>
__device__ __forceinline__ void rollout_body(const MppiRolloutArgs& a) {
  mppi_allow_dependent_launch();
  const uint32_t agent = blockIdx.y, blk = blockIdx.x;
  rollout_item<BLOCK, WS, LANES, EARLY>(a, agent, blk, a.K, a.H, a.u_nom + (size_t)agent * a.H * kM,
                                 a.partials + ((size_t)agent * a.nblk + blk) * a.pstride);
  if (FUSED && a.agent_done)
    fused_combine_tail<WS ? 2 * BLOCK : BLOCK * LANES>(a, agent, a.nblk);
}

// Uneven batch: work items (agent, CTA-of-agent), longest horizons first.
// A persistent grid pulls items from an atomic queue (no CTA ever waits on
// another); without a queue each CTA runs item blockIdx.x.
template <int BLOCK, bool FUSED>
__device__ __forceinline__ void rollout_work(const MppiRolloutArgs& a) {
  __shared__ uint32_t item_s;
  // the work list, K and H are constant over a closed loop; each item waits
  // (griddepcontrol.wait in rollout_item) before it reads the previous
  // launch's results
  mppi_allow_dependent_launch();
  for (uint32_t pass = 0;; ++pass) {
    __syncthreads();  // the previous item is done with shared memory
    if (threadIdx.x == 0)
      item_s = a.work_counter ? atomicAdd(a.work_counter, 1u) : (pass == 0 ? blockIdx.x : ~0u);
    __syncthreads();
    const uint32_t item = item_s;
    if (item >= a.num_work) return;
    const uint2 w = a.work[item];
    const uint32_t agent = w.x, blk = w.y;
    rollout_item<BLOCK>(a, agent, blk, a.agent_K[agent], a.agent_H[agent],
                        a.u_nom + (size_t)agent * a.H * kM,
                        a.partials + ((size_t)a.agent_blk0[agent] + blk) * a.pstride);
    if (FUSED && a.agent_done)
      fused_combine_tail<BLOCK, 0>(a, agent, (a.agent_K[agent] + BLOCK - 1) / BLOCK);
  }
}

// --------------------------------------------------------------------------
// Combine of one agent by a CTA of CB threads: the combine kernel (one CTA
// per agent) or, fused, the agent's last rollout CTA.  Shared memory at dsm:
// scale[nblk] | u[H*m].  The partial records come from other CTAs of this or
// the previous launch and are read through L2 (ld.global.cg).
// --------------------------------------------------------------------------
constexpr int kCombineBlock = 256;

// The propagate's dynamics step x <- f(x, u*_0), compiled once and called by
// every kernel that runs a combine (the combine kernel and the rollout
// kernels' fused tails).  An inlined copy per kernel may contract
// multiply-adds differently in each, and the propagated state -- the next
// step's x0 -- would then depend on the step form chosen for the shape.
// State and control travel by value (registers), not through memory.
struct PropagateState {
  __align__(16) float s[kNPad];
};
struct PropagateControl {
  float u[kM];
};
__device__ __noinline__ PropagateState propagate_dynamics(PropagateState x, PropagateControl c,
                                                          const uint8_t* mp, uint32_t step,
                                                          uint32_t agent) {
  MPPI_DYNAMICS_FN(reinterpret_cast<DynStateT>(reinterpret_cast<void*>(x.s)), c.u, mp,
                   make_uint2(step, 0x80000000u), agent);
  return x;
}

#ifdef MPPI_FEATURES_FN
// The plugin's proposal features f[0, MPPI_MAX_FEATURES) of one state (zero
// where the callable sets none), compiled once for the same reason: the
// features kernel (a loop's first step) and every combine (the steps after
// it) call this one copy, so the network's input -- and with it the proposal
// -- cannot depend on the step form.
__device__ __noinline__ void compute_features(const float* st, const uint8_t* mp,
                                              const uint8_t* cp, float* f) {
#pragma unroll
  for (int i = 0; i < MPPI_MAX_FEATURES; ++i) f[i] = 0.0f;
  MPPI_FEATURES_FN(st, mp, cp, f);
}

// The proposal network for one row, by the calling CTA's threads (all of
// them call it): in -> hidden -> hidden -> hidden -> out with GELU between,
// the features, weights and hidden activations rounded to BF16 and FP32
// accumulation, like the tensor-core kernels.  Output n of a layer belongs
// to threads n, n + blockDim.x, ...; its dot product runs over k in a fixed
// order (four partial sums over k-blocks of 8, blocks b = 0, 1, 2, 3 mod 4,
// added as (s0 + s1) + (s2 + s3)), so the result does not depend on the
// CTA size -- one compiled copy serves the combine kernel, the rollout
// kernels' fused combines and the first step's kernel.  The weights stream
// from L2 in 16-byte pieces of their K-major core-matrix image.
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xffff0000u); }

__device__ __noinline__ void network_row(const float* f, const MppiNetRows& net, float* out) {
  constexpr int kMaxHidden = 256;
  __shared__ __align__(16) float h_s[2][kMaxHidden];
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  for (uint32_t k = tid; k < net.in; k += nt)
    h_s[1][k] = mppi_round_bf16(k < (uint32_t)MPPI_MAX_FEATURES ? f[k] : 0.0f);
  __syncthreads();
  for (int l = 0; l < 4; ++l) {
    const uint32_t K = l == 0 ? net.in : net.hidden;
    const uint32_t N = l == 3 ? net.out : net.hidden;
    const float* hin = h_s[(l + 1) & 1];
    float* hout = h_s[l & 1];
    const uint4* W = reinterpret_cast<const uint4*>(net.w[l]);
    // two outputs per pass (n and n + nt), their weight loads issued in
    // batches of 8 k-blocks each, so 16 loads are in flight per thread (one
    // output: batches of 16 of its k-blocks)
    for (uint32_t n0 = tid; n0 < N; n0 += 2 * nt) {
      const uint32_t n1 = n0 + nt;
      const bool two = n1 < N;
      // row n, k-block b (8 inputs) at element (n / 8) 8K + 64 b + (n % 8) 8
      const uint4* wr0 = W + (size_t)(n0 >> 3) * K + (n0 & 7u);
      const uint4* wr1 = W + (size_t)(n1 >> 3) * K + (n1 & 7u);
      float acc0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, acc1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      const uint32_t nb = K / 8;
      // one k-block (8 inputs) of one output into its partial sum b mod 4
      auto block = [&](float (&acc)[4], const uint4& w, uint32_t b) {
        const float4 h0 = *reinterpret_cast<const float4*>(hin + 8 * b);
        const float4 h1 = *reinterpret_cast<const float4*>(hin + 8 * b + 4);
        float& s = acc[b & 3u];
        s = fmaf(bf16_lo(w.x), h0.x, s);
        s = fmaf(bf16_hi(w.x), h0.y, s);
        s = fmaf(bf16_lo(w.y), h0.z, s);
        s = fmaf(bf16_hi(w.y), h0.w, s);
        s = fmaf(bf16_lo(w.z), h1.x, s);
        s = fmaf(bf16_hi(w.z), h1.y, s);
        s = fmaf(bf16_lo(w.w), h1.z, s);
        s = fmaf(bf16_hi(w.w), h1.w, s);
      };
      // with one output, the second bank of loads holds its next 8 k-blocks
      // (16 in flight either way); the blocks still go in ascending order
      const uint32_t step = two ? 8u : 16u;
      for (uint32_t b0 = 0; b0 < nb; b0 += step) {
        uint4 w0[8], w1[8];
#pragma unroll
        for (uint32_t i = 0; i < 8; ++i) {
          const bool in0 = b0 + i < nb, in1 = two ? in0 : b0 + 8 + i < nb;
          w0[i] = in0 ? __ldg(wr0 + 8 * (b0 + i)) : make_uint4(0u, 0u, 0u, 0u);
          w1[i] = in1 ? __ldg(two ? wr1 + 8 * (b0 + i) : wr0 + 8 * (b0 + 8 + i))
                      : make_uint4(0u, 0u, 0u, 0u);
        }
        if (two) {
#pragma unroll
          for (uint32_t i = 0; i < 8; ++i) {
            if (b0 + i < nb) {
              block(acc0, w0[i], b0 + i);
              block(acc1, w1[i], b0 + i);
            }
          }
        } else {
#pragma unroll
          for (uint32_t i = 0; i < 8; ++i)
            if (b0 + i < nb) block(acc0, w0[i], b0 + i);
#pragma unroll
          for (uint32_t i = 0; i < 8; ++i)
            if (b0 + 8 + i < nb) block(acc0, w1[i], b0 + 8 + i);
        }
      }
      const float z0 = ((acc0[0] + acc0[1]) + (acc0[2] + acc0[3])) + net.b[l][n0];
      if (l < 3)
        hout[n0] = mppi_round_bf16(mppi_gelu(z0));
      else
        out[n0] = z0;
      if (two) {
        const float z1 = ((acc1[0] + acc1[1]) + (acc1[2] + acc1[3])) + net.b[l][n1];
        if (l < 3)
          hout[n1] = mppi_round_bf16(mppi_gelu(z1));
        else
          out[n1] = z1;
      }
    }
    __syncthreads();
  }
}
#endif

// PRE: records whose weighted-sum columns are read ahead (0: none; the
// uneven batches' persistent kernel keeps its registers for the rollout).
template <int CB, uint32_t PRE>
__device__ __forceinline__ void combine_agent(const MppiCombineArgs& a, uint32_t agent,
                                              float* dsm) {
  __shared__ float stat_s[4];
  __shared__ double min_s;
#ifdef MPPI_FEATURES_FN
  __shared__ float feat_s[MPPI_MAX_FEATURES];  // the next step's network input
#if MPPI_CP_SMEM
  // the agent's cost parameters for the feature callable, copied in by all
  // threads at the start (one thread runs the callable, and its reads then
  // hit shared memory instead of L2)
  __shared__ __align__(16) uint32_t fcp_s[(MPPI_CP_BYTES + 3) / 4];
  if (a.features) copy_words(fcp_s, a.cost_params + a.cost_stride * agent, MPPI_CP_BYTES);
#endif
#endif
  const uint32_t tid = threadIdx.x;
  const bool ragged = a.agent_K != nullptr;
  const uint32_t K = ragged ? a.agent_K[agent] : a.K;
  const uint32_t H = ragged ? a.agent_H[agent] : a.H;
  const uint32_t HM = H * kM, ps = a.pstride;
  const uint32_t nblk = ragged ? (K + a.block - 1) / a.block : a.nblk;
  const size_t blk0 = ragged ? (size_t)a.agent_blk0[agent] : (size_t)agent * a.nblk;
  float* scale_s = dsm;
  float* u_s = dsm + ((a.nblk + 3) & ~3u);  // a.nblk: the largest agent's CTA count
  const float* P = a.partials + blk0 * ps;

  float* un = a.u_nom + (size_t)agent * a.H * kM;  // agent stride: the largest horizon
  float* uo = a.u_out + (size_t)agent * a.H * kM;

  // Warp 0's lanes load their first record's head first: the statistics
  // wait on it, so it goes ahead of the reads below in the memory pipeline.
  float h0 = 0.0f, l0 = 0.0f, e0 = 0.0f, q0 = 0.0f, c0 = 0.0f;
  if (tid < 32 && tid < nblk) {
    const float* pb = P + (size_t)tid * ps;
    h0 = ld_early(pb);
    l0 = ld_early(pb + 4);
    e0 = ld_early(pb + 1);
    q0 = ld_early(pb + 2);
    c0 = ld_early(pb + 3);
  }
  // Read ahead, before the statistics are known (one round trip to L2
  // instead of three): each thread's first weighted-sum column of every
  // record and its nominal value (agents of at most PRE records), and the
  // state the propagate stage advances (small states).  Nothing is read
  // ahead with PRE = 0.
  constexpr uint32_t kPre = PRE > 0 ? PRE : 1;
  constexpr bool kPreX = PRE > 0 && kN <= 16;
  const bool pre = PRE > 0 && nblk <= PRE && tid < HM;
  float pv[kPre], un_pre = 0.0f;
  if (pre) {
#pragma unroll
    for (uint32_t b = 0; b < kPre; ++b)
      pv[b] = b < nblk ? ld_early(P + (size_t)b * ps + MPPI_PARTIAL_HEAD + tid) : 0.0f;
    un_pre = ld_early(un + tid);
  }
  float x_pre[kPreX ? kN : 1];
  uint32_t step_pre = 0;
  if (kPreX && tid == 0 && a.propagate) {
#pragma unroll
    for (int d = 0; d < (kPreX ? kN : 1); ++d) x_pre[d] = ld_early(a.x + (size_t)agent * kN + d);
  }
  if (PRE > 0 && tid == 0 && a.propagate) step_pre = *a.step_base + a.step_local;
  // the bounds of this thread's first column (its control dimension)
  const float lo_pre = PRE > 0 && tid < HM ? ld_early(a.u_min + tid % kM) : 0.0f;
  const float hi_pre = PRE > 0 && tid < HM ? ld_early(a.u_max + tid % kM) : 0.0f;

  // Statistics over the CTA records by warp 0 alone (lane l takes records
  // l, l + 32, ...), so the summation order -- and every bit of the result --
  // is the same whichever CTA size runs the combine.
  // The records' minima are cost pairs (hi at 0, lo at 4), compared and
  // subtracted as doubles like the rollout's per-sample costs.  A lane's
  // first record is read once and kept (for up to 32 records, its only one).
  if (tid < 32) {
    double lm = __longlong_as_double(0x7ff0000000000000ll), m0 = lm;
    if (tid < nblk) {
      m0 = cost_pair(h0, l0);
      lm = fmin(lm, m0);
    }
    for (uint32_t b = tid + 32; b < nblk; b += 32) {
      const float* pb = P + (size_t)b * ps;
      lm = fmin(lm, cost_pair(__ldcg(pb), __ldcg(pb + 4)));
    }
    const double Mw = warp_min_d(lm);
    float S = 0.0f, Q = 0.0f, C = 0.0f;
    if (tid < nblk) {
      const float sc = expf(-(float)(m0 - Mw) / a.lambda);
      scale_s[tid] = sc;
      S = fmaf(sc, e0, S);
      Q = fmaf(sc * sc, q0, Q);
      C += c0;
    }
    for (uint32_t b = tid + 32; b < nblk; b += 32) {
      const float* pb = P + (size_t)b * ps;
      const float sc = expf(-(float)(cost_pair(__ldcg(pb), __ldcg(pb + 4)) - Mw) / a.lambda);
      scale_s[b] = sc;
      S = fmaf(sc, __ldcg(pb + 1), S);
      Q = fmaf(sc * sc, __ldcg(pb + 2), Q);
      C += __ldcg(pb + 3);
    }
    S = warp_sum(S);
    Q = warp_sum(Q);
    C = warp_sum(C);
    if (tid == 0) {
      min_s = Mw;
      stat_s[0] = pair_hi(Mw);
      stat_s[1] = S;
      stat_s[2] = Q;
      stat_s[3] = C;
    }
  }
  __syncthreads();  // statistics and scale_s visible
  const float M = stat_s[0], S = stat_s[1], Q = stat_s[2], C = stat_s[3];

  const float invS = 1.0f / S;
  for (uint32_t j = tid; j < HM; j += CB) {
    float v = 0.0f, un_j;
    if (pre && j == tid) {
#pragma unroll
      for (uint32_t b = 0; b < kPre; ++b)  // in record order, as below
        if (b < nblk) v = fmaf(scale_s[b], pv[b], v);
      un_j = un_pre;
    } else {
#pragma unroll 8
      for (uint32_t b = 0; b < nblk; ++b)  // in record order: loads run ahead of the sum
        v = fmaf(scale_s[b], __ldcg(P + (size_t)b * ps + MPPI_PARTIAL_HEAD + j), v);
      un_j = un[j];
    }
    const uint32_t d = j % kM;
    const bool first = PRE > 0 && j == tid;
    const float u = clampf(un_j + v * invS, first ? lo_pre : a.u_min[d],
                           first ? hi_pre : a.u_max[d]);
    u_s[j] = u;
    uo[j] = u;
  }
  if (a.hist_ustar) {
    float* hu = a.hist_ustar + ((size_t)a.step_local * a.num_agents + agent) * a.H * kM;
    for (uint32_t j = tid; j < HM; j += CB) hu[j] = u_s[j];
  }
  if (tid == 0) {
    a.diag[agent * 3 + 0] = M;
    a.diag[agent * 3 + 1] = C / (float)K;
    a.diag[agent * 3 + 2] = S * S / Q;  // 1 / sum w^2 with w = e / S
    if (a.stats) {
      float* st = a.stats + (size_t)agent * MPPI_STATS_STRIDE;
      st[0] = M;
      st[1] = S;
      st[2] = Q;
      st[3] = C;
      st[4] = pair_lo(min_s);
    }
  }
  if (!a.propagate) return;
  __syncthreads();  // u_s complete, all reads of un done

  // ---- propagate & shift (shaders/mppi_reduce.metal:175-231, 413-488) ----
  if (tid == 0) {
    const uint32_t step = PRE > 0 ? step_pre : *a.step_base + a.step_local;
    const uint32_t row = a.step_local * a.num_agents + agent;
    float* xg = a.x + (size_t)agent * kN;
    __align__(16) float st[kNPad];
    float u0[kM];
#pragma unroll
    for (int d = 0; d < kN; ++d) st[d] = kPreX ? x_pre[kPreX ? d : 0] : xg[d];
#pragma unroll
    for (int d = kN; d < kNPad; ++d) st[d] = 0.0f;
#pragma unroll
    for (int d = 0; d < kM; ++d) u0[d] = u_s[d];
    if (a.hist_states)
      for (int d = 0; d < kN; ++d) a.hist_states[(size_t)row * kN + d] = st[d];
    if (a.hist_controls)
      for (int d = 0; d < kM; ++d) a.hist_controls[(size_t)row * kM + d] = u0[d];
    if (a.hist_costs) a.hist_costs[row] = M;
    // counter (step, 0x80000000); seed = agent index (0 for a single agent)
    {
      PropagateState x;
      PropagateControl c;
#pragma unroll
      for (int d = 0; d < kNPad; ++d) x.s[d] = st[d];
#pragma unroll
      for (int d = 0; d < kM; ++d) c.u[d] = u0[d];
      x = propagate_dynamics(x, c, a.model_params + a.model_stride * agent, step, agent);
#pragma unroll
      for (int d = 0; d < kNPad; ++d) st[d] = x.s[d];
    }
#pragma unroll
    for (int d = 0; d < kN; ++d) xg[d] = st[d];
    if (a.terminal)
      for (int d = 0; d < kN; ++d) a.terminal[(size_t)agent * kN + d] = st[d];
#ifdef MPPI_FEATURES_FN
    // the next step's proposal features, from the state just propagated
    if (a.features) {
      float f[MPPI_MAX_FEATURES];
#if MPPI_CP_SMEM
      const uint8_t* fcp = reinterpret_cast<const uint8_t*>(fcp_s);
#else
      const uint8_t* fcp = a.cost_params + a.cost_stride * agent;
#endif
      compute_features(st, a.model_params + a.model_stride * agent, fcp, f);
      float* o = a.features + (size_t)agent * a.feature_stride;
#pragma unroll
      for (int i = 0; i < MPPI_MAX_FEATURES; ++i) {
        if ((uint32_t)i < a.feature_stride) o[i] = f[i];
        feat_s[i] = f[i];
      }
    }
#endif
  }
#ifdef MPPI_FEATURES_FN
  // ... and the next step's network output, by this CTA (the per-agent form)
  if (a.features && a.net.w[0]) {
    __syncthreads();  // feat_s complete
    network_row(feat_s, a.net, a.net.out_buf + (size_t)agent * a.net.out_stride);
  }
#endif
  for (uint32_t j = tid; j < HM; j += CB) {
    const uint32_t t = j / kM, d = j % kM;
    un[j] = (t + 1 < H) ? u_s[j + kM] : u_s[(H - 1) * kM + d];  // shift left, hold last
  }
}

}  // namespace mppi

// Residency is bounded by the noise staging buffer (H*m floats per thread),
// not by registers: 512 resident threads per SM lets the compiler use up to
// 128 registers for instruction-level parallelism.
// mppi_rollout_fused_b<B> carries the combine tail (MppiRolloutArgs::
// agent_done); the backend times both forms on a new shape and keeps the
// faster -- the tail's extra live state can cost some models registers.
#define MPPI_ROLLOUT_ENTRY(B)                                                      \
  extern "C" __global__ void __launch_bounds__(B, 512 / B)                        \
      mppi_rollout_b##B(const MppiRolloutArgs a) {                                \
    mppi::rollout_body<B, false>(a);                                              \
  }                                                                               \
  extern "C" __global__ void __launch_bounds__(B, 512 / B)                        \
      mppi_rollout_fused_b##B(const MppiRolloutArgs a) {                          \
    mppi::rollout_body<B, true>(a);                                               \
  }
MPPI_ROLLOUT_ENTRY(64)
MPPI_ROLLOUT_ENTRY(128)
MPPI_ROLLOUT_ENTRY(256)

// 128-sample forms with the early noise (drawn before the wait for the
// previous launch): launched for uniform batches with the whole horizon
// staged and no proposal output to read.
extern "C" __global__ void __launch_bounds__(128, 4) mppi_rollout_early_b128(const MppiRolloutArgs a) {
  mppi::rollout_body<128, false, false, 1, true>(a);
}
extern "C" __global__ void __launch_bounds__(128, 4)
    mppi_rollout_early_fused_b128(const MppiRolloutArgs a) {
  mppi::rollout_body<128, true, false, 1, true>(a);
}

// Warp-specialised forms for 128-sample CTAs (256 threads: 128 running the
// recurrence, 128 drawing the noise ahead), whole horizon staged.
extern "C" __global__ void __launch_bounds__(256, 2) mppi_rollout_ws_b128(const MppiRolloutArgs a) {
  mppi::rollout_body<128, false, true>(a);
}
extern "C" __global__ void __launch_bounds__(256, 2)
    mppi_rollout_ws_fused_b128(const MppiRolloutArgs a) {
  mppi::rollout_body<128, true, true>(a);
}

// Cooperative forms (plugins with MPPI_STAGE_COST_SPLIT), kCoopLanes threads
// per sample: mppi_rollout_coop32 with 32 samples per CTA (128 threads for
// four lanes), for launches with few CTAs, where it spreads an agent's
// samples over four times as many SMs; mppi_rollout_coop with 128 samples
// per CTA, as many partial records per agent as the one-thread form.
// Without a split the entries exist but the host never launches them
// (mppi_coop_lanes reads 0).
constexpr int kCoopLanesOr1 = mppi::kCoopLanes > 0 ? mppi::kCoopLanes : 1;
extern "C" __device__ const uint32_t mppi_coop_lanes = mppi::kCoopLanes;
extern "C" __global__ void __launch_bounds__(32 * kCoopLanesOr1, 4)
    mppi_rollout_coop32(const MppiRolloutArgs a) {
  if constexpr (mppi::kCoopLanes > 1) mppi::rollout_body<32, false, false, mppi::kCoopLanes, true>(a);
}
extern "C" __global__ void __launch_bounds__(32 * kCoopLanesOr1, 4)
    mppi_rollout_coop32_fused(const MppiRolloutArgs a) {
  if constexpr (mppi::kCoopLanes > 1) mppi::rollout_body<32, true, false, mppi::kCoopLanes, true>(a);
}
extern "C" __global__ void __launch_bounds__(128 * kCoopLanesOr1, 1)
    mppi_rollout_coop(const MppiRolloutArgs a) {
  if constexpr (mppi::kCoopLanes > 1) mppi::rollout_body<128, false, false, mppi::kCoopLanes, true>(a);
}
extern "C" __global__ void __launch_bounds__(128 * kCoopLanesOr1, 1)
    mppi_rollout_coop_fused(const MppiRolloutArgs a) {
  if constexpr (mppi::kCoopLanes > 1) mppi::rollout_body<128, true, false, mppi::kCoopLanes, true>(a);
}

// Uneven batches always use 128-thread CTAs, so the partition of samples into
// CTAs -- and therefore every floating-point sum -- does not depend on the
// tuned grid size or staging mode.
extern "C" __global__ void __launch_bounds__(128, 4) mppi_rollout_work_b128(const MppiRolloutArgs a) {
  mppi::rollout_work<128, false>(a);
}
extern "C" __global__ void __launch_bounds__(128, 4)
    mppi_rollout_work_fused_b128(const MppiRolloutArgs a) {
  mppi::rollout_work<128, true>(a);
}

extern "C" __global__ void __launch_bounds__(mppi::kCombineBlock)
    mppi_combine(const MppiCombineArgs a) {
  extern __shared__ __align__(16) float dsm[];
  mppi::combine_agent<mppi::kCombineBlock, 32>(a, blockIdx.x, dsm);
}

extern "C" __global__ void __launch_bounds__(256) mppi_weights(const MppiWeightsArgs a) {
  const uint32_t agent = blockIdx.y;
  const uint32_t k = blockIdx.x * 256 + threadIdx.x;
  if (k >= a.K) return;
  const float* st = a.stats + (size_t)agent * MPPI_STATS_STRIDE;
  const double M = mppi::cost_pair(st[0], st[4]);
  const size_t i = (size_t)agent * a.K + k;
  const double c = mppi::cost_pair(a.costs[i], a.costs_lo[i]);
  a.weights[i] = expf(-(float)(c - M) / a.lambda) / st[1];
}

extern "C" __global__ void __launch_bounds__(128) mppi_noise(const MppiNoiseArgs a) {
  const uint32_t i = blockIdx.x * 128 + threadIdx.x;
  if (i >= a.count) return;
  float sig[mppi::kSig];
  mppi::load_sigma(a.sigma, sig);
  const uint32_t k = a.k0 + i;
  for (uint32_t t = 0; t < a.H; ++t) {
    float n[2 * mppi::kP], eps[mppi::kM];
    mppi::sample_noise(a.step, a.key, k, a.H, t, sig, n, eps);
    const size_t o = ((size_t)i * a.H + t) * mppi::kM;
#pragma unroll
    for (int d = 0; d < mppi::kM; ++d) {
      if (a.normals) a.normals[o + d] = n[d];
      if (a.eps) a.eps[o + d] = eps[d];
    }
  }
}

#ifdef MPPI_FEATURES_FN
// Proposal features and the per-agent network of state rows: one CTA per
// row (the first step of a loop whose combines evaluate the network).
extern "C" __global__ void __launch_bounds__(128) mppi_proposal_rows(const MppiProposalRowsArgs a) {
  __shared__ float feat_s[MPPI_MAX_FEATURES];
  const uint32_t r = blockIdx.x;
  const MppiFeaturesArgs& fa = a.f;
  // the states come from the previous kernel (no-op in plain launches)
  mppi::mppi_grid_dependency_wait();
  if (a.given_features) {
    if (threadIdx.x < (uint32_t)MPPI_MAX_FEATURES)
      feat_s[threadIdx.x] =
          threadIdx.x < fa.out_stride ? fa.out[(size_t)r * fa.out_stride + threadIdx.x] : 0.0f;
  } else if (threadIdx.x == 0) {
    const uint32_t agent = r % fa.agents_mod;
    __align__(16) float st[mppi::kNPad];
    const float* xr = fa.x + (size_t)r * fa.x_stride;
#pragma unroll
    for (int d = 0; d < mppi::kN; ++d) st[d] = xr[d];
#pragma unroll
    for (int d = mppi::kN; d < mppi::kNPad; ++d) st[d] = 0.0f;
    float f[MPPI_MAX_FEATURES];
    mppi::compute_features(st, fa.model_params + fa.model_stride * agent,
                           fa.cost_params + fa.cost_stride * agent, f);
#pragma unroll
    for (int i = 0; i < MPPI_MAX_FEATURES; ++i) feat_s[i] = f[i];
    if (fa.out) {
      float* o = fa.out + (size_t)r * fa.out_stride;
#pragma unroll
      for (int i = 0; i < MPPI_MAX_FEATURES; ++i)
        if ((uint32_t)i < fa.out_stride) o[i] = f[i];
    }
  }
  __syncthreads();
  mppi::network_row(feat_s, a.net, a.net.out_buf + (size_t)r * a.net.out_stride);
}

// Proposal features: one thread per state row.
extern "C" __global__ void __launch_bounds__(128) mppi_features(const MppiFeaturesArgs a) {
  const uint32_t r = blockIdx.x * 128 + threadIdx.x;
  if (r >= a.rows) return;
  const uint32_t agent = r % a.agents_mod;
  __align__(16) float st[mppi::kNPad];
  const float* xr = a.x + (size_t)r * a.x_stride;
#pragma unroll
  for (int d = 0; d < mppi::kN; ++d) st[d] = xr[d];
#pragma unroll
  for (int d = mppi::kN; d < mppi::kNPad; ++d) st[d] = 0.0f;
  float f[MPPI_MAX_FEATURES];
  mppi::compute_features(st, a.model_params + a.model_stride * agent,
                         a.cost_params + a.cost_stride * agent, f);
  float* o = a.out + (size_t)r * a.out_stride;
#pragma unroll
  for (int i = 0; i < MPPI_MAX_FEATURES; ++i)
    if ((uint32_t)i < a.out_stride) o[i] = f[i];
}
#endif
