// proposal_mlp.cu — the learned sampling proposal: a 4-layer MLP
// (in -> 256 -> 256 -> 256 -> H*m + m, GELU) with BF16 weights and
// activations and FP32 accumulation on the sm_100a tensor cores (tcgen05,
// accumulators in TMEM), trained with its own backward and Adam kernels.
//
// Kernels
//   mlp_fused   one CTA (512 threads) per 128 batch rows.  Forward: 4 GEMMs, each an
//               A (activations, 128 x K) x B (weights, N x K) product issued
//               as K/16 tcgen05.mma instructions by one thread into a
//               128 x N FP32 TMEM accumulator; the weights arrive by bulk
//               copy while the previous layer's epilogue runs, the epilogue
//               (bias, GELU, BF16) writes the next layer's A operand straight
//               into shared memory.  Training continues in the same CTA
//               with the loss (Gaussian NLL of u*) and three more GEMMs for
//               the activation gradients dH = dZ W, saving for the weight
//               gradients dZ^T and H^T (batch-contiguous images).
//   mlp_forward_cluster   inference: a cluster of 8 CTAs per 128 rows, each
//               computing an eighth of every layer's output columns and
//               broadcasting its slice of the activations into the other
//               CTAs' shared memory (DSMEM), so the MMAs, epilogues and
//               weight loads of one tile are spread over 8 SMs.
//   mlp_wgrad   dW_l = dZ_l^T H_{l-1} summed over the batch: split over
//               batch chunks, a 4-stage bulk-copy ring feeding the MMAs,
//               FP32 atomics into the gradient.
//   mlp_bgrad   db_l = column sums of dZ_l.
//   mlp_adam    Adam on FP32 master weights; rewrites the BF16 operand
//               images W (rows = outputs) and W^T (rows = inputs).
//
// Shared-memory operand layout: K-major core-matrix tiles (tc_sm100.cuh):
//   canon(r, k; K) = (r/8) * 8K + (k/8) * 64 + (r%8) * 8 + k%8   [elements]
// i.e. LBO = 128 B, SBO = 16 K bytes.  Global weight images use the same
// layout, so one bulk copy lands a whole matrix ready for the MMA.  Batch-
// contiguous images ("T-images", operands of the weight-gradient GEMM) hold
// a matrix of R rows over the batch in 64-column chunks, each chunk a
// canonical R x 64 tile (LBO = 128 B, SBO = 1024 B):
//   timg(r, col; R) = (col/64) * 64R + (r/8) * 512 + ((col%64)/8) * 64 + (r%8) * 8 + col%8
//
// Every wait is bounded (tc::kWaitCycles); a wait that gives up sets a bit
// of the error word, the CTA skips the remaining work, waits (bounded) for
// its copies in flight and frees its TMEM.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/mppi_b200/mppi_backend.h"
#include "../../include/mppi_b200/mppi_proposal.h"
#include "device/mppi_gelu.cuh"
#include "device/tc_sm100.cuh"
#include "proposal.hpp"

namespace mppi_b200 {
namespace prop {

using bf16 = __nv_bfloat16;

constexpr uint32_t kTile = 128;  // batch rows per CTA = TMEM lanes
// mlp_fused runs kGroups warps per TMEM lane quarter: warp w reads lanes
// 32 (w % 4) .. +31 (its rows) and handles the 16-column chunks
// j = w / 4 (mod kGroups) of every epilogue.
constexpr uint32_t kGroups = 4;
constexpr uint32_t kFusedThreads = kTile * kGroups;
constexpr uint32_t kHid = 256;   // hidden width
constexpr uint32_t kIn = 32;     // padded input width
constexpr uint32_t kMaxM = 16;   // control dims handled by the loss epilogue
constexpr uint32_t kTmemCols = 256;

// mlp_fused shared memory: A tile | W tile | barriers | loss scratch
constexpr uint32_t kSmemA = kTile * kHid * 2;   // 64 KB
constexpr uint32_t kSmemW = kHid * kHid * 2;    // 128 KB
constexpr uint32_t kSmemBar = 64;
constexpr uint32_t kSmemLoss = 3 * kMaxM * kTile * 4;  // 24 KB
constexpr uint32_t kFusedSmem = kSmemA + kSmemW + kSmemBar + kSmemLoss;

// mlp_wgrad shared memory: kStages x (A 128 x 64 | B <= 256 x 64) | barriers
constexpr uint32_t kStages = 4;
constexpr uint32_t kStageA = kTile * 64 * 2;  // 16 KB
constexpr uint32_t kStageB = kHid * 64 * 2;   // 32 KB
constexpr uint32_t kWgradSmem = kStages * (kStageA + kStageB) + 128;

static_assert(kFusedSmem <= 232448, "fused kernel exceeds the shared-memory limit");
static_assert(kWgradSmem <= 232448, "wgrad kernel exceeds the shared-memory limit");

__host__ __device__ __forceinline__ uint32_t canon(uint32_t r, uint32_t k, uint32_t kdim) {
  return (r >> 3) * (kdim * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

__host__ __device__ __forceinline__ size_t timg(uint32_t r, uint32_t col, uint32_t rows) {
  return (size_t)(col >> 6) * rows * 64 + (r >> 3) * 512 + ((col & 63) >> 3) * 64 + (r & 7) * 8 +
         (col & 7);
}

// GELU and its derivative (csrc/device/mppi_gelu.cuh: erf by Abramowitz and
// Stegun 7.1.26 on the SM's reciprocal and exp2), shared with the per-agent
// network evaluation of the MPPI module.
__device__ __forceinline__ float gelu(float z) { return mppi_gelu(z); }

__device__ __forceinline__ float gelu_grad(float z) {
  float cdf, g;
  mppi_gelu_phi(z, cdf, g);
  return fmaf(z * 0.39894228040143268f, g, cdf);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Row t, columns [16j, 16j + 16) of a canonical A tile of contraction kdim.
__device__ __forceinline__ void a_store16(bf16* as, uint32_t t, uint32_t j, uint32_t kdim,
                                          const float (&v)[16]) {
  const uint32_t base = canon(t, 16 * j, kdim);
  *reinterpret_cast<uint4*>(as + base) =
      make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]), pack2(v[6], v[7]));
  *reinterpret_cast<uint4*>(as + base + 64) = make_uint4(
      pack2(v[8], v[9]), pack2(v[10], v[11]), pack2(v[12], v[13]), pack2(v[14], v[15]));
}

// Rows [r0, r0 + 16) of column `col` of a T-image with `rows` rows.
__device__ __forceinline__ void t_store16(bf16* img, uint32_t rows, uint32_t col, uint32_t r0,
                                          const float (&v)[16]) {
  bf16* p = img + timg(0, col, rows);
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const uint32_t r = r0 + i;
    p[(r >> 3) * 512 + (r & 7) * 8] = __float2bfloat16_rn(v[i]);
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Bulk copy of `bytes` (multiple of 16) in 32 KB pieces, completing on bar.
__device__ __forceinline__ void load_operand(uint32_t dst, const void* src, uint32_t bytes,
                                             uint32_t bar) {
  tc::mbar_expect_tx(bar, bytes);
  const char* s = static_cast<const char*>(src);
  for (uint32_t off = 0; off < bytes; off += 32768u)
    tc::bulk_g2s(dst + off, s + off, min(32768u, bytes - off), bar);
}

// ---------------------------------------------------------------------------
// mlp_fused
// ---------------------------------------------------------------------------
struct FusedArgs {
  const bf16* W[4];   // forward B operands: rows = outputs, contraction = inputs
  const bf16* WT[4];  // backward B operands (1..3): rows = inputs, contraction = outputs
  const float* b[4];
  const float* x;
  const float* target;
  const uint32_t* index;
  float* out;
  float* z[3];     // pre-activations [mp][256]
  bf16* hT[4];     // layer inputs, T-images (rows 32, 256, 256, 256)
  bf16* dzT[4];    // output gradients, T-images (rows 256)
  float* loss;
  int* err;
  uint32_t x_stride, target_stride, out_stride, rows, mp;
  uint32_t in_dim, out_dim, out_pad, hm, m, train;
  float ls_min, ls_max, inv_norm;
};

// GEMM g of the fused kernel: 0..3 forward layers, 4..6 activation
// gradients through layers 3, 2, 1.
__device__ __forceinline__ uint32_t gemm_k(uint32_t g, uint32_t out_pad) {
  return g == 0 ? kIn : (g == 4 ? out_pad : kHid);
}
__device__ __forceinline__ uint32_t gemm_n(uint32_t g, uint32_t out_pad) {
  return g == 3 ? out_pad : kHid;
}
__device__ __forceinline__ const bf16* gemm_b(const FusedArgs& a, uint32_t g) {
  return g < 4 ? a.W[g] : a.WT[7 - g];
}

__global__ void __launch_bounds__(kFusedThreads, 1) mlp_fused_kernel(const FusedArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  bf16* as = reinterpret_cast<bf16*>(smem);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kSmemA + kSmemW);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2);
  volatile uint32_t* abort_s = tslot + 1;
  float* lsc_s = reinterpret_cast<float*>(smem + kSmemA + kSmemW + kSmemBar);  // [d][128]
  float* iv_s = lsc_s + kMaxM * kTile;
  float* gls_s = iv_s + kMaxM * kTile;

  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t quarter = warp & 3u, grp = warp >> 2;
  const uint32_t r = quarter * 32 + lane;  // this thread's row of the tile
  const uint32_t row = blockIdx.x * kTile + r;
  const bool valid = row < a.rows;
  const uint32_t bar_w = tc::smem_addr(&bars[0]), bar_m = tc::smem_addr(&bars[1]);
  const uint32_t a_s = tc::smem_addr(as), w_s = a_s + kSmemA;

  if (tid == 0) {
    tc::mbar_init(bar_w, 1);
    tc::mbar_init(bar_m, 1);
    *abort_s = 0;
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_addr(tslot), kTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t t_row = tmem + ((quarter * 32u) << 16);

  bool w_pending = false;
  uint32_t ph_w = 0, ph_m = 0;
  if (tid == 0) {
    load_operand(w_s, a.W[0], kHid * kIn * 2, bar_w);
    w_pending = true;
  }

  // ---- input row -> A (contraction 32); training keeps x^T for dW0 ----
  const uint32_t src = valid ? (a.index ? a.index[row] : row) : 0u;
#pragma unroll
  for (uint32_t j = grp; j < kIn / 16; j += kGroups) {
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint32_t c = 16 * j + i;
      v[i] = (valid && c < a.in_dim) ? a.x[(size_t)src * a.x_stride + c] : 0.0f;
    }
    a_store16(as, r, j, kIn, v);
    if (a.train) t_store16(a.hT[0], kIn, row, 16 * j, v);
  }

  const uint32_t n_gemm = a.train ? 7u : 4u;
  for (uint32_t g = 0; g < n_gemm; ++g) {
    const uint32_t K = gemm_k(g, a.out_pad), N = gemm_n(g, a.out_pad);
    // ---- B operand resident, A written: issue the K/16 MMAs ----
    if (tid == 0) {
      if (tc::mbar_wait(bar_w, ph_w)) {
        w_pending = false;
        ph_w ^= 1u;
      } else {
        atomicOr(a.err, 1);
        *abort_s = 1;
      }
    }
    tc::fence_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    if (*abort_s) break;
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t idesc = tc::idesc_bf16(kTile, N);
      const uint32_t sbo = K * 16;
      for (uint32_t s = 0; s < K / 16; ++s)
        tc::mma_bf16(tmem, tc::sdesc(a_s + s * 256, 128, sbo), tc::sdesc(w_s + s * 256, 128, sbo),
                     idesc, s > 0 ? 1u : 0u);
      tc::mma_commit(bar_m);
    }
    const bool done = tc::mbar_wait(bar_m, ph_m);
    ph_m ^= 1u;
    if (__syncthreads_or(!done)) {
      if (tid == 0) atomicOr(a.err, 2);
      break;
    }
    tc::fence_after_sync();
    // ---- the next B operand streams in while this epilogue runs ----
    if (tid == 0 && g + 1 < n_gemm) {
      const uint32_t g1 = g + 1;
      load_operand(w_s, gemm_b(a, g1), gemm_n(g1, a.out_pad) * gemm_k(g1, a.out_pad) * 2, bar_w);
      w_pending = true;
    }

    if (g < 3) {
      // hidden layer g: z = acc + b; h = GELU(z) -> A of layer g + 1
      const float* bias = a.b[g];
      for (uint32_t j = grp; j < kHid / 16; j += kGroups) {
        float v[16];
        tc::tmem_ld16(t_row + 16 * j, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] += bias[16 * j + i];
        if (a.train) {
          float4* zp = reinterpret_cast<float4*>(a.z[g] + (size_t)row * kHid + 16 * j);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            zp[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = gelu(v[i]);
        a_store16(as, r, j, kHid, v);
        if (a.train) t_store16(a.hT[g + 1], kHid, row, 16 * j, v);
      }
    } else if (g == 3 && !a.train) {
      // output layer (inference): out = acc + b
      const float* bias = a.b[3];
      for (uint32_t j = grp; j < a.out_pad / 16; j += kGroups) {
        float v[16];
        tc::tmem_ld16(t_row + 16 * j, v);
        if (valid) {
          float* o = a.out + (size_t)row * a.out_stride + 16 * j;
#pragma unroll
          for (int i = 0; i < 16; ++i) o[i] = v[i] + bias[16 * j + i];
        }
      }
    } else if (g == 3) {
      // output layer (training): loss and dL/d(out) -> A of GEMM 4 and dZ3^T
      // (one warp per lane quarter: the log-scale gradient sums a whole row)
      if (grp == 0) {
      const float* bias = a.b[3];
      const uint32_t m = a.m, hm = a.hm;
      uint32_t inside = 0;
      for (uint32_t d = 0; d < m; ++d) {
        const float raw = tc::tmem_ld1(t_row + hm + d) + bias[hm + d];
        const float c = fminf(fmaxf(raw, a.ls_min), a.ls_max);
        lsc_s[d * kTile + r] = c;
        iv_s[d * kTile + r] = expf(-2.0f * c);
        gls_s[d * kTile + r] = 0.0f;
        if (raw > a.ls_min && raw < a.ls_max) inside |= 1u << d;
      }
      const float* tg = a.target + (size_t)src * a.target_stride;
      float lrow = 0.0f;
      uint32_t d = 0;  // c mod m while c < hm
      for (uint32_t j = 0; j < a.out_pad / 16; ++j) {
        float v[16];
        tc::tmem_ld16(t_row + 16 * j, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const uint32_t c = 16 * j + i;
          float gv = 0.0f;
          if (valid && c < a.out_dim) {
            if (c < hm) {
              const float diff = tg[c] - (v[i] + bias[c]);
              const float iv = iv_s[d * kTile + r];
              lrow += 0.5f * diff * diff * iv + lsc_s[d * kTile + r];
              gv = -diff * iv * a.inv_norm;
              gls_s[d * kTile + r] += (1.0f - diff * diff * iv) * a.inv_norm;
            } else {
              const uint32_t e = c - hm;
              gv = ((inside >> e) & 1u) ? gls_s[e * kTile + r] : 0.0f;
            }
          }
          if (c < hm) d = (d + 1 == m) ? 0u : d + 1;
          v[i] = gv;
        }
        a_store16(as, r, j, a.out_pad, v);
        t_store16(a.dzT[3], kHid, row, 16 * j, v);
      }
      const float s = warp_sum(lrow * a.inv_norm);
      if (lane == 0) atomicAdd(a.loss, s);
      }
    } else {
      // activation gradient through layer 7 - g: dZ = dH * GELU'(z)
      const uint32_t l = 6 - g;
      const float* zr = a.z[l] + (size_t)row * kHid;
      for (uint32_t j = grp; j < kHid / 16; j += kGroups) {
        float v[16];
        tc::tmem_ld16(t_row + 16 * j, v);
        const float4* zp = reinterpret_cast<const float4*>(zr + 16 * j);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 zz = zp[q];
          v[4 * q] *= gelu_grad(zz.x);
          v[4 * q + 1] *= gelu_grad(zz.y);
          v[4 * q + 2] *= gelu_grad(zz.z);
          v[4 * q + 3] *= gelu_grad(zz.w);
        }
        if (g < 6) a_store16(as, r, j, kHid, v);
        t_store16(a.dzT[l], kHid, row, 16 * j, v);
      }
    }
  }

  if (tid == 0 && w_pending && !tc::mbar_wait(bar_w, ph_w)) atomicOr(a.err, 4);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// mlp_forward_cluster: inference, 8 CTAs (one cluster) per 128-row tile
// ---------------------------------------------------------------------------
constexpr uint32_t kCluster = 8;
constexpr uint32_t kCThreads = kTile * kGroups;        // 512
constexpr uint32_t kCSmemW = 32 * kHid * 2;            // this CTA's weight rows (<= 32)
constexpr uint32_t kBiasFloats = 3 * kHid + kHid;       // b0..b2 and b3 (<= 256)
constexpr uint32_t kClusterSmem = 2 * kSmemA + kCSmemW + kSmemBar + kBiasFloats * 4;
constexpr uint32_t kCTmemCols = 32;
static_assert(kClusterSmem <= 232448, "cluster kernel exceeds the shared-memory limit");

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
  uint32_t out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(saddr), "r"(rank));
  return out;
}
// Every thread of every CTA of the cluster arrives; all pass together.
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// 16-column chunks of an N-wide layer dealt to the cluster's CTAs (the MMA's
// N is a multiple of 16): 32 columns each of a 256-wide hidden layer.
__device__ __forceinline__ void cluster_slice(uint32_t N, uint32_t c, uint32_t& col0,
                                              uint32_t& ncols) {
  const uint32_t chunks = N / 16, q = chunks / kCluster, rem = chunks % kCluster;
  col0 = 16 * (c * q + min(c, rem));
  ncols = 16 * (q + (c < rem ? 1u : 0u));
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint4 v) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v.x), "r"(v.y),
               "r"(v.z), "r"(v.w)
               : "memory");
}

// Remote asynchronous store: 16 bytes into another CTA's shared memory,
// counted on that CTA's mbarrier (complete_tx) -- the async proxy, like a
// bulk copy, so the receiving tensor core may read the data once the
// barrier's phase completes, with no proxy fence or cluster barrier.
__device__ __forceinline__ void st_async_v4(uint32_t addr, uint4 v, uint32_t mbar) {
  asm volatile(
      "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, "
      "[%5];" ::"r"(addr),
      "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(mbar)
      : "memory");
}

// Activations ping-pong between two A tiles, each with its own "full"
// mbarrier: layer g reads A[g % 2]; its epilogue stores the CTA's column
// slice of the next activations into its own A[(g + 1) % 2] with plain
// stores and into the seven peers' with st.async, completing 56 KB per layer
// on each receiver's full barrier, which the receiver arms (arrive.expect_tx)
// and waits on before its next MMA.  Reuse is safe by causality: a CTA writes A[(g + 1) % 2] of a peer
// only after its own MMA g, which needed that peer's slice of layer g's
// input, which the peer sent after its MMA g - 1 -- the last reader of the
// buffer being overwritten -- had completed.  Only the start (every
// barrier initialised before any remote arrival) and the end (no CTA
// leaves while a peer may still write into it) synchronise the cluster.
__global__ void __cluster_dims__(kCluster, 1, 1) __launch_bounds__(kCThreads, 1)
    mlp_forward_cluster_kernel(const FusedArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  bf16* as0 = reinterpret_cast<bf16*>(smem);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * kSmemA + kCSmemW);
  // bars: [0] weights, [1] MMA, [2..3] full A[0] / A[1]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 4);
  volatile uint32_t* abort_s = tslot + 1;
  float* bias_s = reinterpret_cast<float*>(smem + 2 * kSmemA + kCSmemW + kSmemBar);  // [4][256]

  const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t quarter = warp & 3u, grp = warp >> 2;
  const uint32_t r = quarter * 32 + lane;
  const uint32_t crank = cluster_rank();
  for (uint32_t i = tid; i < kBiasFloats; i += kCThreads) {
    const uint32_t l = i / kHid, n = i % kHid;
    bias_s[i] = (l < 3 || n < a.out_pad) ? a.b[l][n] : 0.0f;
  }
  const uint32_t row = (blockIdx.x / kCluster) * kTile + r;
  const bool valid = row < a.rows;
  const uint32_t bar_w = tc::smem_addr(&bars[0]), bar_m = tc::smem_addr(&bars[1]);
  const uint32_t bar_full0 = tc::smem_addr(&bars[2]);
  const uint32_t a_s0 = tc::smem_addr(as0), w_s = a_s0 + 2 * kSmemA;
  constexpr uint32_t kTileBytes = kTile * kHid * 2;  // one exchanged activation tile

  if (tid == 0) {
    for (uint32_t i = 0; i < 4; ++i) tc::mbar_init(bar_w + 8 * i, 1);
    *abort_s = 0;
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_addr(tslot), kCTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;
  const uint32_t t_row = tmem + ((quarter * 32u) << 16);
  cluster_sync_all();  // every CTA's barriers exist before any remote arrival

  bool w_pending = false;
  uint32_t ph_w = 0, ph_m = 0, ph_f[2] = {0, 0};
  {
    uint32_t c0, nc;
    cluster_slice(kHid, crank, c0, nc);
    if (tid == 0 && nc) {
      load_operand(w_s, a.W[0] + (size_t)c0 * kIn, nc * kIn * 2, bar_w);
      w_pending = true;
    }
  }
  // the features come from the previous kernel (programmatic launches run
  // everything above while it finishes; a no-op otherwise)
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // input rows -> A[0] (every CTA stages the whole tile itself)
#pragma unroll
  for (uint32_t j = grp; j < kIn / 16; j += kGroups) {
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const uint32_t c = 16 * j + i;
      v[i] = (valid && c < a.in_dim) ? a.x[(size_t)row * a.x_stride + c] : 0.0f;
    }
    a_store16(as0, r, j, kIn, v);
  }

  for (uint32_t g = 0; g < 4; ++g) {
    const uint32_t K = g == 0 ? kIn : kHid, N = g == 3 ? a.out_pad : kHid;
    uint32_t col0, nc;
    cluster_slice(N, crank, col0, nc);
    const uint32_t buf = g & 1u;
    // The next kernel (the rollout that reads this output) may be scheduled
    // from the last layer on: it runs its loop-constant prologue meanwhile.
    // Not earlier -- its CTAs would land on SMs still busy with the kernel
    // before this one and crowd those that free up first.
    if (g == 3) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint32_t a_in = a_s0 + buf * kSmemA;
    if (tid == 0) {
      // weights of this layer, then (past layer 0) the exchanged input tile
      if (w_pending) {
        if (tc::mbar_wait(bar_w, ph_w)) {
          w_pending = false;
          ph_w ^= 1u;
        } else {
          atomicOr(a.err, 1);
          *abort_s = 1;
        }
      }
      if (g > 0) {
        // the peers' column slices of layer g - 1's output (this CTA's own
        // slice was stored locally)
        const uint32_t full = bar_full0 + 8 * buf;
        uint32_t oc0, onc;
        cluster_slice(kHid, crank, oc0, onc);
        tc::mbar_expect_tx(full, kTileBytes - kTile * onc * 2);
        if (!tc::mbar_wait(full, ph_f[buf])) {
          atomicOr(a.err, 8);
          *abort_s = 1;
        }
        ph_f[buf] ^= 1u;
      }
    }
    tc::fence_async_shared();
    tc::fence_before_sync();
    __syncthreads();
    const bool run = !*abort_s && nc > 0;
    if (run && tid == 0) {
      tc::fence_after_sync();
      const uint32_t idesc = tc::idesc_bf16(kTile, nc);
      const uint32_t sbo = K * 16;
      for (uint32_t s2 = 0; s2 < K / 16; ++s2)
        tc::mma_bf16(tmem, tc::sdesc(a_in + s2 * 256, 128, sbo),
                     tc::sdesc(w_s + s2 * 256, 128, sbo), idesc, s2 > 0 ? 1u : 0u);
      tc::mma_commit(bar_m);
    }
    bool done = true;
    if (run) {
      done = tc::mbar_wait(bar_m, ph_m);
      ph_m ^= 1u;
    }
    if (__syncthreads_or(!done)) {
      if (tid == 0) {
        atomicOr(a.err, 2);
        *abort_s = 1;
      }
      __syncthreads();
    }
    tc::fence_after_sync();
    const bool ok = run && !*abort_s;
    // the next layer's weight rows stream in during this epilogue
    if (tid == 0 && g < 3 && !*abort_s) {
      uint32_t c1, n1;
      cluster_slice(g == 2 ? a.out_pad : kHid, crank, c1, n1);
      if (n1) {
        load_operand(w_s, a.W[g + 1] + (size_t)c1 * kHid, n1 * kHid * 2, bar_w);
        w_pending = true;
      }
    }
    if (ok && g < 3) {
      // h = GELU(acc + b) for this CTA's columns -> A[(g + 1) % 2] of every CTA
      const float* bias = bias_s + g * kHid + col0;
      const uint32_t nbuf = (g + 1) & 1u;
      const uint32_t off = a_s0 + nbuf * kSmemA;
      const uint32_t full = bar_full0 + 8 * nbuf;
      // 8-column pieces: a warp's 32 rows x 8 columns, one 16-byte core-matrix
      // row (8 BF16) per thread, so all four warps of a lane quarter work
      for (uint32_t j = grp; j < nc / 8; j += kGroups) {
        float v[8];
        tc::tmem_ld8(t_row + 8 * j, v);
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = gelu(v[i] + bias[8 * j + i]);
        const uint4 h8 = make_uint4(pack2(v[0], v[1]), pack2(v[2], v[3]), pack2(v[4], v[5]),
                                    pack2(v[6], v[7]));
        const uint32_t dst = off + 2 * canon(r, col0 + 8 * j, kHid);
        // this CTA's own slice by plain local stores (made visible to the
        // tensor core by the proxy fence and barrier at the next layer's
        // start), the peers' copies by remote asynchronous stores
        st_shared_v4(dst, h8);
#pragma unroll
        for (uint32_t q = 1; q < kCluster; ++q) {
          const uint32_t peer = (crank + q) % kCluster;
          st_async_v4(map_to_rank(dst, peer), h8, map_to_rank(full, peer));
        }
      }
    } else if (ok) {
      // output layer: this CTA's columns straight to global memory
      const float* bias = bias_s + 3 * kHid + col0;
      for (uint32_t j = grp; j < nc / 8; j += kGroups) {
        float v[8];
        tc::tmem_ld8(t_row + 8 * j, v);
        if (valid) {
          float* o = a.out + (size_t)row * a.out_stride + col0 + 8 * j;
#pragma unroll
          for (int i = 0; i < 8; ++i) o[i] = v[i] + bias[8 * j + i];
        }
      }
    }
  }

  if (tid == 0 && w_pending && !tc::mbar_wait(bar_w, ph_w)) atomicOr(a.err, 4);
  tc::fence_before_sync();
  cluster_sync_all();  // no CTA leaves while a peer may still store into it
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kCTmemCols);
  }
}

// ---------------------------------------------------------------------------
// mlp_wgrad: gW_l[n][k] += sum over the batch of dZ_l[., n] H_{l-1}[., k]
// grid (splits, 4 layers x 2 row tiles), 128 threads
// ---------------------------------------------------------------------------
struct WgradArgs {
  const bf16* dzT[4];
  const bf16* hT[4];
  float* gW[4];
  uint32_t rows_out[4];  // output rows of W_l
  uint32_t kdim[4];      // input width of W_l (= rows of hT_l)
  uint32_t chunks;       // 64-column batch chunks
  uint32_t splits;
  int* err;
};

__global__ void __launch_bounds__(128, 1) mlp_wgrad_kernel(const WgradArgs a) {
  const uint32_t l = blockIdx.y >> 1, rt = blockIdx.y & 1u;
  const uint32_t c0 = blockIdx.x * a.chunks / a.splits;
  const uint32_t c1 = (blockIdx.x + 1) * a.chunks / a.splits;
  if (rt * kTile >= a.rows_out[l] || c0 >= c1) return;  // uniform per CTA

  extern __shared__ __align__(128) uint8_t smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kStages * (kStageA + kStageB));
  // bars: full[kStages] | empty[kStages] | done | tmem slot
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 1);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const uint32_t s_base = tc::smem_addr(smem);
  const uint32_t bar0 = tc::smem_addr(bars);
  auto full = [&](uint32_t s) { return bar0 + 8 * s; };
  auto empty = [&](uint32_t s) { return bar0 + 8 * (kStages + s); };
  const uint32_t done_bar = bar0 + 8 * (2 * kStages);

  if (tid == 0) {
    for (uint32_t s = 0; s < 2 * kStages + 1; ++s) tc::mbar_init(bar0 + 8 * s, 1);
    tc::mbar_init_fence();
  }
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_addr(tslot), kTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tslot;

  const uint32_t K = a.kdim[l];
  const uint32_t bytes_b = K * 64 * 2;
  const bf16* a_img = a.dzT[l] + (size_t)rt * kTile * 64;  // + chunk * 256 * 64
  const bf16* b_img = a.hT[l];                             // + chunk * K * 64
  const uint32_t n = c1 - c0;

  if (tid == 0) {
    uint32_t issued[kStages] = {0, 0, 0, 0}, used[kStages] = {0, 0, 0, 0};
    auto issue = [&](uint32_t i, uint32_t st) {
      const uint32_t c = c0 + i;
      tc::mbar_expect_tx(full(st), kStageA + bytes_b);
      tc::bulk_g2s(s_base + st * kStageA, a_img + (size_t)c * kHid * 64, kStageA, full(st));
      tc::bulk_g2s(s_base + kStages * kStageA + st * kStageB, b_img + (size_t)c * K * 64,
                   bytes_b, full(st));
      ++issued[st];
    };
    bool ok = true;
    for (uint32_t i = 0; i < n && i < kStages; ++i) issue(i, i);
    const uint32_t idesc = tc::idesc_bf16(kTile, K);
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t st = i % kStages;
      if (!tc::mbar_wait(full(st), (i / kStages) & 1u)) {
        ok = false;
        break;
      }
      ++used[st];
      tc::fence_after_sync();
      const uint32_t sa = s_base + st * kStageA, sb = s_base + kStages * kStageA + st * kStageB;
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k)
        tc::mma_bf16(tmem, tc::sdesc(sa + k * 256, 128, 1024), tc::sdesc(sb + k * 256, 128, 1024),
                     idesc, (i > 0 || k > 0) ? 1u : 0u);
      tc::mma_commit(empty(st));
      // refill the stage chunk i - 1 used, once its MMAs are done
      if (i >= 1 && i - 1 + kStages < n) {
        const uint32_t sp = (i - 1) % kStages;
        if (!tc::mbar_wait(empty(sp), ((i - 1) / kStages) & 1u)) {
          ok = false;
          break;
        }
        issue(i - 1 + kStages, sp);
      }
    }
    tc::mma_commit(done_bar);
    if (!ok) {
      atomicOr(a.err, 8);
      // drain copies that were issued but never consumed
      for (uint32_t st = 0; st < kStages; ++st)
        for (uint32_t q = used[st]; q < issued[st]; ++q) tc::mbar_wait(full(st), q & 1u);
    }
  }
  const bool done = tc::mbar_wait(done_bar, 0);
  if (__syncthreads_or(!done)) {
    if (tid == 0) atomicOr(a.err, 16);
  } else {
    tc::fence_after_sync();
    const uint32_t nrow = rt * kTile + tid;
    const uint32_t t_row = tmem + ((warp * 32u) << 16);
    float* gw = a.gW[l] + (size_t)nrow * K;
    for (uint32_t j = 0; j < K / 16; ++j) {
      float v[16];
      tc::tmem_ld16(t_row + 16 * j, v);
      if (nrow < a.rows_out[l]) {
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(gw + 16 * j + i, v[i]);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTmemCols);
  }
}

// ---------------------------------------------------------------------------
// mlp_bgrad: gb_l[n] = sum over the batch of dZ_l[., n]; one warp per row
// ---------------------------------------------------------------------------
struct BgradArgs {
  const bf16* dzT[4];
  float* gb[4];
  uint32_t rows_out[4];
  uint32_t mp;
};

__global__ void __launch_bounds__(256) mlp_bgrad_kernel(const BgradArgs a) {
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  const uint32_t l = gw / kHid, n = gw % kHid;
  if (l >= 4 || n >= a.rows_out[l]) return;
  const bf16* img = a.dzT[l];
  float s = 0.0f;
  for (uint32_t p = lane; p < a.mp / 8; p += 32) {
    const uint32_t mc = p >> 3, cc = p & 7u;
    const uint4 q = *reinterpret_cast<const uint4*>(img + (size_t)mc * kHid * 64 + (n >> 3) * 512 +
                                                    cc * 64 + (n & 7) * 8);
    const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float2 f = __bfloat1622float2(h[i]);
      s += f.x + f.y;
    }
  }
  s = warp_sum(s);
  if (lane == 0) a.gb[l][n] = s;
}

// ---------------------------------------------------------------------------
// mlp_adam: Adam step on the FP32 master parameters (update != 0) and the
// BF16 operand images of the weights
// ---------------------------------------------------------------------------
struct AdamArgs {
  float* p;
  const float* g;
  float* m1;
  float* m2;
  uint64_t count;
  uint64_t seg[9];  // starts of W0 b0 W1 b1 W2 b2 W3 b3, end
  uint32_t rows[4];
  uint32_t kdim[4];
  bf16* W[4];
  bf16* WT[4];
  float lr_t, beta1, beta2, eps;
  uint32_t update;
};

__global__ void __launch_bounds__(256) mlp_adam_kernel(const AdamArgs a) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.count;
       i += (uint64_t)gridDim.x * blockDim.x) {
    float w = a.p[i];
    if (a.update) {
      const float g = a.g[i];
      const float m = a.beta1 * a.m1[i] + (1.0f - a.beta1) * g;
      const float v = a.beta2 * a.m2[i] + (1.0f - a.beta2) * g * g;
      a.m1[i] = m;
      a.m2[i] = v;
      w -= a.lr_t * m / (sqrtf(v) + a.eps);
      a.p[i] = w;
    }
    uint32_t s = 0;
    while (s < 7 && i >= a.seg[s + 1]) ++s;
    if ((s & 1u) == 0) {
      const uint32_t l = s >> 1;
      const uint32_t off = (uint32_t)(i - a.seg[s]);
      const uint32_t nn = off / a.kdim[l], kk = off % a.kdim[l];
      const bf16 h = __float2bfloat16_rn(w);
      a.W[l][canon(nn, kk, a.kdim[l])] = h;
      if (l >= 1) a.WT[l][canon(kk, nn, a.rows[l])] = h;
    }
  }
}

}  // namespace prop
}  // namespace mppi_b200

// ===========================================================================
// Host object
// ===========================================================================
using namespace mppi_b200::prop;

struct mppi_proposal {
  mppi_proposal_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint32_t hm = 0, out_dim = 0, out_pad = 0;
  uint32_t rows[4] = {kHid, kHid, kHid, 0};
  uint32_t kdim[4] = {kIn, kHid, kHid, kHid};
  uint64_t seg[9] = {};
  uint64_t count = 0;
  float* params = nullptr;  // device: params | grads | m1 | m2 (count each)
  float* grads = nullptr;
  float* m1 = nullptr;
  float* m2 = nullptr;
  bf16* wimg = nullptr;     // device: W0..W3 images then WT1..WT3 images
  bf16* W[4] = {};
  bf16* WT[4] = {};
  // training buffers, capacity cap_mp batch rows
  uint32_t cap_mp = 0;
  float* z = nullptr;
  bf16* himg = nullptr;
  bf16* dzimg = nullptr;
  float* loss_d = nullptr;  // [0] loss, [1] error word
  float* loss_h = nullptr;  // pinned copy
  int64_t adam_t = 0;
  float last_ms = 0.0f;
};

namespace {

void set_err(char* err, size_t len, const std::string& msg) {
  if (err && len) {
    const size_t k = msg.size() < len - 1 ? msg.size() : len - 1;
    memcpy(err, msg.data(), k);
    err[k] = '\0';
  }
}

int cuda_fail(cudaError_t e, const char* what, char* err, size_t len) {
  set_err(err, len, std::string(what) + ": " + cudaGetErrorString(e));
  return MPPI_ERR_CUDA;
}

#define PROP_CUDA(call, what)                                \
  do {                                                       \
    const cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, what, err, err_len); \
  } while (0)

// splitmix64 -> uniform [-1, 1)
struct InitRng {
  uint64_t s;
  float next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (float)((double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0);
  }
};

int* err_word(mppi_proposal* p) { return reinterpret_cast<int*>(p->loss_d + 1); }

int refresh_images(mppi_proposal* p, bool update, float lr, char* err, size_t err_len) {
  AdamArgs a{};
  a.p = p->params;
  a.g = p->grads;
  a.m1 = p->m1;
  a.m2 = p->m2;
  a.count = p->count;
  for (int i = 0; i < 9; ++i) a.seg[i] = p->seg[i];
  for (int l = 0; l < 4; ++l) {
    a.rows[l] = p->rows[l];
    a.kdim[l] = p->kdim[l];
    a.W[l] = p->W[l];
    a.WT[l] = p->WT[l];
  }
  a.beta1 = 0.9f;
  a.beta2 = 0.999f;
  a.eps = 1e-8f;
  a.update = update ? 1u : 0u;
  if (update) {
    ++p->adam_t;
    const double t = (double)p->adam_t;
    a.lr_t = (float)(lr * std::sqrt(1.0 - std::pow(0.999, t)) / (1.0 - std::pow(0.9, t)));
  }
  mlp_adam_kernel<<<592, 256, 0, p->stream>>>(a);
  PROP_CUDA(cudaGetLastError(), "adam launch");
  return MPPI_OK;
}

int ensure_train_buffers(mppi_proposal* p, uint32_t mp, char* err, size_t err_len) {
  if (mp <= p->cap_mp) return MPPI_OK;
  cudaFree(p->z);
  cudaFree(p->himg);
  cudaFree(p->dzimg);
  p->z = nullptr;
  p->himg = nullptr;
  p->dzimg = nullptr;
  p->cap_mp = 0;
  PROP_CUDA(cudaMalloc(&p->z, (size_t)3 * mp * kHid * 4), "cudaMalloc");
  PROP_CUDA(cudaMalloc(&p->himg, (size_t)(kIn + 3 * kHid) * mp * 2), "cudaMalloc");
  PROP_CUDA(cudaMalloc(&p->dzimg, (size_t)4 * kHid * mp * 2), "cudaMalloc");
  // rows of the output-gradient image past the output width stay zero
  PROP_CUDA(cudaMemsetAsync(p->dzimg, 0, (size_t)4 * kHid * mp * 2, p->stream), "cudaMemset");
  p->cap_mp = mp;
  return MPPI_OK;
}

// forward + loss + backward (+ Adam when lr >= 0 and `step`)
int run_train(mppi_proposal* p, const float* x, uint32_t x_stride, const float* target,
              uint32_t target_stride, const uint32_t* index, uint32_t rows, bool step, float lr,
              float* loss_out, float* grads_host, char* err, size_t err_len) {
  if (!x || !target || rows == 0 || x_stride < p->cfg.input_dim || target_stride < p->hm) {
    set_err(err, err_len, "proposal training: null input, zero rows or a stride below the row width.");
    return MPPI_ERR_INVALID;
  }
  if (rows > p->cfg.max_batch) {
    set_err(err, err_len, "proposal training: rows exceed max_batch.");
    return MPPI_ERR_INVALID;
  }
  PROP_CUDA(cudaSetDevice(p->device), "cudaSetDevice");
  const uint32_t tiles = (rows + kTile - 1) / kTile;
  const uint32_t mp = tiles * kTile;
  if (int rc = ensure_train_buffers(p, mp, err, err_len)) return rc;
  const size_t mpz = (size_t)mp * kHid;

  PROP_CUDA(cudaEventRecord(p->ev0, p->stream), "event");
  PROP_CUDA(cudaMemsetAsync(p->grads, 0, p->count * 4, p->stream), "cudaMemset");
  PROP_CUDA(cudaMemsetAsync(p->loss_d, 0, 4, p->stream), "cudaMemset");  // loss; not the error word

  FusedArgs f{};
  for (int l = 0; l < 4; ++l) {
    f.W[l] = p->W[l];
    f.WT[l] = p->WT[l];
    f.b[l] = p->params + p->seg[2 * l + 1];
  }
  f.x = x;
  f.target = target;
  f.index = index;
  f.out = nullptr;
  for (int l = 0; l < 3; ++l) f.z[l] = p->z + l * mpz;
  f.hT[0] = p->himg;
  for (int l = 1; l < 4; ++l) f.hT[l] = p->himg + (size_t)kIn * mp + (size_t)(l - 1) * kHid * mp;
  for (int l = 0; l < 4; ++l) f.dzT[l] = p->dzimg + (size_t)l * kHid * mp;
  f.loss = p->loss_d;
  f.err = err_word(p);
  f.x_stride = x_stride;
  f.target_stride = target_stride;
  f.out_stride = 0;
  f.rows = rows;
  f.mp = mp;
  f.in_dim = p->cfg.input_dim;
  f.out_dim = p->out_dim;
  f.out_pad = p->out_pad;
  f.hm = p->hm;
  f.m = p->cfg.control_dim;
  f.train = 1;
  f.ls_min = p->cfg.log_scale_min;
  f.ls_max = p->cfg.log_scale_max;
  f.inv_norm = 1.0f / ((float)rows * (float)p->hm);
  mlp_fused_kernel<<<tiles, kFusedThreads, kFusedSmem, p->stream>>>(f);
  PROP_CUDA(cudaGetLastError(), "mlp_fused launch");

  WgradArgs w{};
  for (int l = 0; l < 4; ++l) {
    w.dzT[l] = f.dzT[l];
    w.hT[l] = f.hT[l];
    w.gW[l] = p->grads + p->seg[2 * l];
    w.rows_out[l] = p->rows[l];
    w.kdim[l] = p->kdim[l];
  }
  w.chunks = mp / 64;
  w.splits = std::max(1u, std::min(w.chunks, 18u));
  w.err = err_word(p);
  mlp_wgrad_kernel<<<dim3(w.splits, 8), 128, kWgradSmem, p->stream>>>(w);
  PROP_CUDA(cudaGetLastError(), "mlp_wgrad launch");

  BgradArgs bg{};
  for (int l = 0; l < 4; ++l) {
    bg.dzT[l] = f.dzT[l];
    bg.gb[l] = p->grads + p->seg[2 * l + 1];
    bg.rows_out[l] = p->rows[l];
  }
  bg.mp = mp;
  mlp_bgrad_kernel<<<(4 * kHid * 32 + 255) / 256, 256, 0, p->stream>>>(bg);
  PROP_CUDA(cudaGetLastError(), "mlp_bgrad launch");

  if (step)
    if (int rc = refresh_images(p, true, lr, err, err_len)) return rc;
  PROP_CUDA(cudaEventRecord(p->ev1, p->stream), "event");

  if (grads_host)
    PROP_CUDA(cudaMemcpyAsync(grads_host, p->grads, p->count * 4, cudaMemcpyDeviceToHost,
                              p->stream),
              "cudaMemcpy");
  PROP_CUDA(cudaMemcpyAsync(p->loss_h, p->loss_d, 8, cudaMemcpyDeviceToHost, p->stream),
            "cudaMemcpy");
  if (loss_out || grads_host || !step) {
    PROP_CUDA(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
    cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1);
    int ew;
    memcpy(&ew, p->loss_h + 1, 4);
    if (ew != 0) {
      cudaMemset(p->loss_d + 1, 0, 4);
      set_err(err, err_len, "proposal kernels: a bounded wait gave up (error word " +
                                std::to_string(ew) + ").");
      return MPPI_ERR_CUDA;
    }
    if (loss_out) *loss_out = p->loss_h[0];
  }
  return MPPI_OK;
}

}  // namespace

namespace mppi_b200 {

ProposalShape proposal_shape(const mppi_proposal* p) {
  return ProposalShape{p->cfg.input_dim, p->cfg.horizon, p->cfg.control_dim, p->out_pad,
                       p->cfg.log_scale_min, p->cfg.log_scale_max, p->device};
}

ProposalWeights proposal_weights(const mppi_proposal* p) {
  ProposalWeights w{};
  for (int l = 0; l < 4; ++l) {
    w.w[l] = reinterpret_cast<const uint16_t*>(p->W[l]);
    w.b[l] = p->params + p->seg[2 * l + 1];
  }
  w.in = kIn;
  w.hidden = kHid;
  w.out = p->out_pad;
  return w;
}

cudaError_t proposal_enqueue_forward(mppi_proposal* p, cudaStream_t stream, const float* x,
                                     uint32_t x_stride, uint32_t rows, float* out,
                                     bool programmatic) {
  if (rows == 0) return cudaSuccess;
  FusedArgs f{};
  for (int l = 0; l < 4; ++l) {
    f.W[l] = p->W[l];
    f.WT[l] = p->WT[l];
    f.b[l] = p->params + p->seg[2 * l + 1];
  }
  f.x = x;
  f.out = out;
  f.err = err_word(p);
  f.x_stride = x_stride;
  f.out_stride = p->out_pad;
  f.rows = rows;
  f.mp = ((rows + kTile - 1) / kTile) * kTile;
  f.in_dim = p->cfg.input_dim;
  f.out_dim = p->out_dim;
  f.out_pad = p->out_pad;
  f.hm = p->hm;
  f.m = p->cfg.control_dim;
  f.train = 0;
  if (!programmatic) {
    mlp_forward_cluster_kernel<<<(f.mp / kTile) * kCluster, kCThreads, kClusterSmem, stream>>>(f);
    return cudaGetLastError();
  }
  // may start while the previous kernel finishes: the kernel sets up TMEM,
  // barriers, biases and the first weights, then waits for that grid before
  // it reads the features
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((f.mp / kTile) * kCluster);
  cfg.blockDim = dim3(kCThreads);
  cfg.dynamicSmemBytes = kClusterSmem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, mlp_forward_cluster_kernel, f);
}

bool proposal_check_device_error(mppi_proposal* p, std::string* msg) {
  int ew = 0;
  if (cudaMemcpy(&ew, p->loss_d + 1, 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
    if (msg) *msg = "proposal: reading the device error word failed.";
    return false;
  }
  if (ew == 0) return true;
  cudaMemset(p->loss_d + 1, 0, 4);
  if (msg) *msg = "proposal kernels: a bounded wait gave up (error word " + std::to_string(ew) + ").";
  return false;
}

}  // namespace mppi_b200

extern "C" {

mppi_proposal* mppi_proposal_create(const mppi_proposal_config* c, char* err, size_t err_len) {
  if (!c) {
    set_err(err, err_len, "null proposal config.");
    return nullptr;
  }
  if (c->input_dim == 0 || c->input_dim > kIn || c->horizon == 0 || c->control_dim == 0 ||
      c->control_dim > kMaxM || (uint64_t)c->horizon * c->control_dim + c->control_dim > kHid ||
      c->max_batch == 0 || !(c->log_scale_min < c->log_scale_max)) {
    set_err(err, err_len,
            "proposal config: need 1 <= input_dim <= 32, control_dim <= 16, "
            "horizon*control_dim + control_dim <= 256, max_batch >= 1, "
            "log_scale_min < log_scale_max.");
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    set_err(err, err_len, "No CUDA device available.");
    return nullptr;
  }
  mppi_proposal* p = new (std::nothrow) mppi_proposal();
  if (!p) return nullptr;
  p->cfg = *c;
  cudaGetDevice(&p->device);
  p->hm = c->horizon * c->control_dim;
  p->out_dim = p->hm + c->control_dim;
  p->out_pad = (p->out_dim + 15) / 16 * 16;
  p->rows[3] = p->out_pad;
  uint64_t off = 0;
  for (int l = 0; l < 4; ++l) {
    p->seg[2 * l] = off;
    off += (uint64_t)p->rows[l] * p->kdim[l];
    p->seg[2 * l + 1] = off;
    off += p->rows[l];
  }
  p->seg[8] = off;
  p->count = off;

  auto fail = [&](const char* what, cudaError_t e) -> mppi_proposal* {
    set_err(err, err_len, std::string(what) + ": " + cudaGetErrorString(e));
    mppi_proposal_destroy(p);
    return nullptr;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail("cudaStreamCreate", e);
  if ((e = cudaEventCreate(&p->ev0)) != cudaSuccess || (e = cudaEventCreate(&p->ev1)) != cudaSuccess)
    return fail("cudaEventCreate", e);
  if ((e = cudaMalloc(&p->params, p->count * 4 * 4)) != cudaSuccess) return fail("cudaMalloc", e);
  p->grads = p->params + p->count;
  p->m1 = p->grads + p->count;
  p->m2 = p->m1 + p->count;
  size_t img = 0;
  for (int l = 0; l < 4; ++l) img += (size_t)p->rows[l] * p->kdim[l];
  for (int l = 1; l < 4; ++l) img += (size_t)p->rows[l] * p->kdim[l];
  if ((e = cudaMalloc(&p->wimg, img * 2)) != cudaSuccess) return fail("cudaMalloc", e);
  size_t o = 0;
  for (int l = 0; l < 4; ++l) {
    p->W[l] = p->wimg + o;
    o += (size_t)p->rows[l] * p->kdim[l];
  }
  for (int l = 1; l < 4; ++l) {
    p->WT[l] = p->wimg + o;
    o += (size_t)p->rows[l] * p->kdim[l];
  }
  if ((e = cudaMalloc(&p->loss_d, 16)) != cudaSuccess) return fail("cudaMalloc", e);
  if ((e = cudaMallocHost(&p->loss_h, 16)) != cudaSuccess) return fail("cudaMallocHost", e);
  if ((e = cudaFuncSetAttribute(mlp_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kFusedSmem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(mlp_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kWgradSmem)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(mlp_forward_cluster_kernel,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kClusterSmem)) !=
          cudaSuccess)
    return fail("cudaFuncSetAttribute", e);

  // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), output layer x 0.1
  std::vector<float> h(p->count, 0.0f);
  InitRng rng{c->seed};
  for (int l = 0; l < 4; ++l) {
    const uint32_t fan_in = l == 0 ? c->input_dim : kHid;
    const uint32_t valid_rows = l == 3 ? p->out_dim : kHid;
    const float bound = (l == 3 ? 0.1f : 1.0f) / std::sqrt((float)fan_in);
    for (uint32_t n = 0; n < valid_rows; ++n)
      for (uint32_t k = 0; k < fan_in; ++k)
        h[p->seg[2 * l] + (uint64_t)n * p->kdim[l] + k] = bound * rng.next();
    for (uint32_t n = 0; n < valid_rows; ++n) h[p->seg[2 * l + 1] + n] = bound * rng.next();
  }
  char tmp[256];
  if (mppi_proposal_set_params(p, h.data(), p->count, tmp, sizeof tmp) != MPPI_OK) {
    set_err(err, err_len, tmp);
    mppi_proposal_destroy(p);
    return nullptr;
  }
  return p;
}

void mppi_proposal_destroy(mppi_proposal* p) {
  if (!p) return;
  cudaSetDevice(p->device);
  if (p->stream) cudaStreamSynchronize(p->stream);
  cudaFree(p->params);
  cudaFree(p->wimg);
  cudaFree(p->z);
  cudaFree(p->himg);
  cudaFree(p->dzimg);
  cudaFree(p->loss_d);
  if (p->loss_h) cudaFreeHost(p->loss_h);
  if (p->ev0) cudaEventDestroy(p->ev0);
  if (p->ev1) cudaEventDestroy(p->ev1);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

uint64_t mppi_proposal_param_count(const mppi_proposal* p) { return p ? p->count : 0; }

uint32_t mppi_proposal_output_stride(const mppi_proposal* p) { return p ? p->out_pad : 0; }

float mppi_proposal_last_train_ms(const mppi_proposal* p) { return p ? p->last_ms : 0.0f; }

int mppi_proposal_set_params(mppi_proposal* p, const float* params_host, uint64_t count,
                             char* err, size_t err_len) {
  if (!p || !params_host || count != p->count) {
    set_err(err, err_len, "set_params: null argument or count != param_count.");
    return MPPI_ERR_INVALID;
  }
  PROP_CUDA(cudaSetDevice(p->device), "cudaSetDevice");
  PROP_CUDA(cudaMemcpyAsync(p->params, params_host, count * 4, cudaMemcpyHostToDevice, p->stream),
            "cudaMemcpy");
  PROP_CUDA(cudaMemsetAsync(p->grads, 0, 3 * count * 4, p->stream), "cudaMemset");  // grads, moments
  PROP_CUDA(cudaMemsetAsync(p->loss_d, 0, 16, p->stream), "cudaMemset");
  p->adam_t = 0;
  if (int rc = refresh_images(p, false, 0.0f, err, err_len)) return rc;
  PROP_CUDA(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
  return MPPI_OK;
}

int mppi_proposal_get_params(mppi_proposal* p, float* params_host, uint64_t count, char* err,
                             size_t err_len) {
  if (!p || !params_host || count != p->count) {
    set_err(err, err_len, "get_params: null argument or count != param_count.");
    return MPPI_ERR_INVALID;
  }
  PROP_CUDA(cudaSetDevice(p->device), "cudaSetDevice");
  PROP_CUDA(cudaMemcpyAsync(params_host, p->params, count * 4, cudaMemcpyDeviceToHost, p->stream),
            "cudaMemcpy");
  PROP_CUDA(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
  return MPPI_OK;
}

int mppi_proposal_forward(mppi_proposal* p, const float* x_dev, uint32_t x_stride, uint32_t rows,
                          float* out_dev, char* err, size_t err_len) {
  if (!p || !x_dev || !out_dev || x_stride < (p ? p->cfg.input_dim : 0)) {
    set_err(err, err_len, "forward: null argument or x_stride below input_dim.");
    return MPPI_ERR_INVALID;
  }
  PROP_CUDA(cudaSetDevice(p->device), "cudaSetDevice");
  PROP_CUDA(mppi_b200::proposal_enqueue_forward(p, p->stream, x_dev, x_stride, rows, out_dev),
            "mlp_fused launch");
  PROP_CUDA(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
  std::string msg;
  if (!mppi_b200::proposal_check_device_error(p, &msg)) {
    set_err(err, err_len, msg);
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}

int mppi_proposal_gradients(mppi_proposal* p, const float* x_dev, uint32_t x_stride,
                            const float* target_dev, uint32_t target_stride,
                            const uint32_t* index_dev, uint32_t rows, float* loss_out,
                            float* grads_host, char* err, size_t err_len) {
  if (!p) {
    set_err(err, err_len, "null proposal.");
    return MPPI_ERR_INVALID;
  }
  return run_train(p, x_dev, x_stride, target_dev, target_stride, index_dev, rows, false, 0.0f,
                   loss_out, grads_host, err, err_len);
}

int mppi_proposal_train_step(mppi_proposal* p, const float* x_dev, uint32_t x_stride,
                             const float* target_dev, uint32_t target_stride,
                             const uint32_t* index_dev, uint32_t rows, float learning_rate,
                             float* loss_out, char* err, size_t err_len) {
  if (!p || !(learning_rate >= 0.0f)) {
    set_err(err, err_len, "train_step: null proposal or negative learning rate.");
    return MPPI_ERR_INVALID;
  }
  return run_train(p, x_dev, x_stride, target_dev, target_stride, index_dev, rows, true,
                   learning_rate, loss_out, nullptr, err, err_len);
}

}  // extern "C"
