// backend.cpp — the CUDA backend behind include/mppi_b200/mppi_backend.h.
//
// Host side of the hot path: owns the per-driver kernel module (NVRTC), the
// CUDA stream, device buffers and pinned staging buffers, chooses the launch
// geometry and the form of a step, and issues the step's launches (captured
// into a CUDA graph for closed loops).  Replaces the reference's MetalBackend
// (src/metal_backend.mm): there, one command buffer per call encodes four
// passes per step with buffer barriers and waits for completion; here each
// control step is one rollout launch whose agents' last CTAs also combine
// (or a rollout and a combine kernel, whichever form the per-shape timing
// keeps), a T-step closed loop is one graph launch, and the host waits once
// per call.
//   done      [N] u32          finished rollout CTAs per agent (fused combine)
//
// Device data layout for a batch of N agents (all FP32, agent-major):
//   io:       [step_base u32 x4][x N*n][u_nom N*H*m][u_out N*H*m][diag N*3]
//             [stats N*MPPI_STATS_STRIDE]
//             (step_base..u_nom is one upload, u_out..diag one download)
//   costs     [N][K] hi, [N][K] lo  per-sample cost pairs of the last single
//                               control step (dispatch_rollout); the closed
//                               loops do not write them
//   partials  [N][nblk][ps]     per-CTA softmax / weighted-noise partials
//   history   [T][N][n], [T][N][m], [T][N]; terminal [N][n]
//   per-agent blobs [N][pad16(size)], per-agent sigma [N][m or m*m]
#include "../../include/mppi_b200/mppi_backend.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "device/mppi_launch.h"
#include "proposal.hpp"
#include "nvrtc_module.hpp"

namespace {

using mppi_b200::KernelModule;

void set_err(char* err, size_t len, const std::string& msg) {
  if (err != nullptr && len > 0) {
    const size_t n = std::min(len - 1, msg.size());
    memcpy(err, msg.data(), n);
    err[n] = '\0';
  }
}

size_t pad4(size_t n) { return (n + 3) & ~size_t(3); }
size_t pad16(size_t n) { return (n + 15) & ~size_t(15); }

constexpr uint32_t kFeatureStride = 32;  // floats per feature row (network input)
// Batches of at most this many agents evaluate the proposal network per agent
// inside their combines (CUDA cores, weights streamed from L2); larger ones
// run the tensor-core batch kernel, which reads the weights once per 128
// agents (MPPI_B200_NET_PER_AGENT=0 / 1 pins the choice).
constexpr uint32_t kNetPerAgentMax = 512;

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // Returns true when the buffer was (re)allocated.
  cudaError_t ensure(size_t n, bool* grew = nullptr) {
    if (n == 0) n = 16;
    if (p && n <= bytes) return cudaSuccess;
    release();
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) bytes = n;
    if (grew) *grew = true;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t ensure(size_t n) {
    if (n == 0) n = 16;
    if (p && n <= bytes) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, n);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Cholesky factor of a row-major SPD matrix (lower triangle), in double.
bool cholesky(uint32_t m, const float* a, std::vector<float>* l) {
  std::vector<double> L((size_t)m * m, 0.0);
  for (uint32_t i = 0; i < m; ++i) {
    for (uint32_t j = 0; j <= i; ++j) {
      double s = a[i * m + j];
      for (uint32_t k = 0; k < j; ++k) s -= L[i * m + k] * L[j * m + k];
      if (i == j) {
        if (!(s > 0.0)) return false;
        L[i * m + i] = std::sqrt(s);
      } else {
        L[i * m + j] = s / L[j * m + j];
      }
    }
  }
  l->assign(L.begin(), L.end());
  return true;
}

struct LaunchGeom {
  int variant = 1;  // index into kRolloutBlocks
  uint32_t block = 128;  // samples per CTA
  uint32_t nblk = 0;
  uint32_t stage_rows = 0;
  uint32_t pstride = 0;
  size_t smem = 0;
  // cooperative form: lanes per sample (0: one thread per sample); its CTAs
  // have block * coop threads; coop_v indexes the module's cooperative
  // entries (0: 32 samples per CTA, 1: 128)
  uint32_t coop = 0;
  int coop_v = 1;
};

}  // namespace

struct mppi_backend {
  // ---- configuration (fixed at initialize) ----
  bool initialized = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint32_t n = 0, m = 0, H = 0, K = 0;
  float lambda = 1.0f;
  bool cov_full = false;
  bool control_cost = false;
  bool noise_half = false;   // NumericMode kFp16 / kMixed
  size_t stage_elem = 4;     // bytes per staged noise value
  uint32_t seed = 0;
  uint64_t mp_size = 0, cp_size = 0;
  std::vector<float> sigma_dev;  // std-devs (diag) or Cholesky factor (full)
  std::vector<float> sigma_inv;
  std::vector<float> u_min, u_max;
  std::shared_ptr<const KernelModule> mod;
  mppi_b200::ModuleSpec spec;  // what `mod` was compiled from
  int num_sms = 148;
  size_t max_smem_optin = 0;
  size_t smem_per_sm = 233472;   // shared memory of one SM
  size_t smem_reserved = 1024;   // reserved by the system in every CTA

  // ---- constant device data ----
  DevBuf d_consts;  // [sigma m*m][sigma_inv m*m][u_min m][u_max m] padded
  DevBuf d_mp_bound, d_cp_bound, d_mp_ovr, d_cp_ovr, d_zero;
  bool mp_bound = false, cp_bound = false;

  // ---- per-shape state ----
  uint32_t N = 0, T = 0;
  LaunchGeom geom;
  DevBuf d_io, d_costs, d_partials;
  DevBuf d_done;  // [N] per-agent count of finished rollout CTAs (fused combine)
  // false: never run the combine inside the rollout launch (its agent's last
  // CTA) -- MPPI_B200_SEPARATE_COMBINE=1
  bool fuse_combine = true;
  // MPPI_B200_FUSED_COMBINE=1 / MPPI_B200_WS=1 or 0 pin the step form's
  // combine and warp-specialisation choices (0 = timed)
  int combine_pin = 0, ws_pin = 0;
  // MPPI_B200_COOP=1 / 0 pins the cooperative form on / off (0 = the shape
  // rule of choose_geometry)
  int coop_pin = 0;
  // MPPI_B200_NO_EARLY_NOISE=1: the 128-sample one-thread forms draw their
  // noise after the grid wait (the same bits; for comparisons)
  bool no_early = false;
  // MPPI_B200_NET_PER_AGENT=1 / 0 pins the proposal network's form (0 = by
  // the batch size, kNetPerAgentMax)
  int net_pin = 0;
  uint32_t form = 0;          // for form_key's launch shape: kFormFused | kFormWs
  std::string form_key;
  // Uniform rollout launches (and the proposal network's) use programmatic
  // dependent launch; MPPI_B200_NO_PDL=1 launches them plainly.
  bool pdl = true;
  DevBuf d_hs, d_hc, d_hk, d_term;
  DevBuf d_agent_sigma, d_agent_mp, d_agent_cp;
  bool want_s = false, want_c = false, want_k = false, want_t = false;
  // parameter pointers of the prepared run
  const uint8_t* run_mp = nullptr;
  const uint8_t* run_cp = nullptr;
  uint64_t run_mp_stride = 0, run_cp_stride = 0;
  const float* run_sigma = nullptr;
  uint32_t run_sigma_stride = 0;
  uint64_t generation = 0;  // bumps whenever a device buffer is reallocated

  PinnedBuf h_up, h_down;
  bool run_timed = false;  // ev0 / ev1 bracket the last closed-loop run

  // ---- uneven batch (per-agent K and H) ----
  bool ragged = false;
  std::vector<uint32_t> agent_K, agent_H, agent_blk0;
  uint32_t num_work = 0;     // work items (agent, CTA-of-agent)
  uint32_t total_records = 0;
  uint32_t grid = 0;         // persistent grid size; 0 = one CTA per item
  DevBuf d_agent_info;       // [K N][H N][blk0 N] uint32
  DevBuf d_work;             // [num_work] uint2, longest horizons first
  DevBuf d_queue;            // atomic work counter
  std::string tuned_key;
  float tuned_ms = 0.0f;
  LaunchGeom tuned_geom;     // the autotuner's choice for tuned_key
  uint32_t tuned_grid = 0;

  // ---- learned proposal ----
  uint32_t feature_dim = 0;            // features per row (plugin callable)
  mppi_proposal* proposal = nullptr;   // attached network (not owned)
  uint32_t prop_samples = 0;           // samples per agent drawn from it
  DevBuf d_feat;                       // [N][32] features of the current states
  DevBuf d_prop;                       // [N][out_stride] network outputs
  bool record_ustar = false;
  DevBuf d_hu;                         // [T][N][H*m] u* of every closed-loop step

  // ---- closed-loop graph cache ----
  cudaGraphExec_t graph = nullptr;
  std::string graph_key;
  // one control step (dispatch_rollout): uploads, kernels, download
  cudaGraphExec_t step_graph = nullptr;
  std::string step_key;
  std::string shape_key;  // shape of the last ensure_shape (uniform batches)

  ~mppi_backend() {
    if (graph) cudaGraphExecDestroy(graph);
    if (step_graph) cudaGraphExecDestroy(step_graph);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }

  size_t sig_len() const { return cov_full ? (size_t)m * m : m; }
  size_t HM() const { return (size_t)H * m; }

  // io buffer offsets (floats)
  size_t off_x() const { return 4; }
  size_t off_unom() const { return off_x() + pad4((size_t)N * n); }
  size_t off_uout() const { return off_unom() + pad4((size_t)N * HM()); }
  size_t off_diag() const { return off_uout() + pad4((size_t)N * HM()); }
  size_t off_stats() const { return off_diag() + pad4((size_t)N * 3); }
  size_t io_floats() const { return off_stats() + (size_t)N * MPPI_STATS_STRIDE; }

  float* io() const { return d_io.as<float>(); }
  const float* c_sigma() const { return d_consts.as<float>(); }
  const float* c_sigma_inv() const { return d_consts.as<float>() + pad4((size_t)m * m); }
  const float* c_umin() const { return d_consts.as<float>() + 2 * pad4((size_t)m * m); }
  const float* c_umax() const { return c_umin() + pad4(m); }
};

namespace {

// Dynamic shared memory one rollout CTA may use so that four fit on an SM.
size_t rollout_dynamic_share(const mppi_backend* b, size_t static_smem, size_t budget) {
  const size_t quarter = b->smem_per_sm / 4;
  const size_t overhead = b->smem_reserved + static_smem;
  const size_t share = quarter > overhead + 4096 ? quarter - overhead : 4096;
  return std::min(share, budget);
}

// Shared memory of a rollout CTA in front of the noise staging: the nominal
// sequence, plus the proposal's mean shift in modules compiled for one.
size_t nominal_bytes(const mppi_backend* b) {
  return pad4(b->HM()) * 4 * (b->spec.proposal ? 2 : 1);
}

#define CK(call)                                                                      \
  do {                                                                                \
    cudaError_t _e = (call);                                                          \
    if (_e != cudaSuccess) {                                                          \
      set_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(_e) +     \
                                " (" #call ")");                                     \
      return (_e == cudaErrorNoDevice || _e == cudaErrorInsufficientDriver)           \
                 ? MPPI_ERR_NO_DEVICE                                                 \
                 : MPPI_ERR_CUDA;                                                     \
    }                                                                                 \
  } while (0)

bool valid_identifier(const char* s) {
  if (!s || !*s) return false;
  for (const char* c = s; *c; ++c) {
    const bool ok = (*c == '_') || (*c >= 'a' && *c <= 'z') || (*c >= 'A' && *c <= 'Z') ||
                    (c != s && *c >= '0' && *c <= '9');
    if (!ok) return false;
  }
  return true;
}

// Launch geometry for N agents (fixed K, H): block size and how the noise
// is kept for the weighted sums.  Staging the whole horizon during the
// rollout avoids regenerating it; it needs H*m*block*4 bytes per CTA, so it
// is used while that keeps four CTAs per SM, or when every CTA of the launch
// is resident at once with it; otherwise the noise is regenerated in chunks
// after the costs are known.
// The cooperative form (the plugin's stage cost split over lanes, module
// coop_lanes > 0) serves launches whose one-thread form would have at most
// one 128-sample CTA per four SMs (a single agent, a few agents): there each
// sample's serial chain sets the time, and splitting its cost terms over
// lanes, with 32-sample CTAs spread over four times as many SMs, shortens it
// (the single-agent configuration: 13.9 against 15.5 us per control step).
// With more CTAs the SMs' issue slots fill and the lanes' repeated dynamics
// only add work (2.4x the instructions; the proposal workload's 256 CTAs ran
// 25% slower cooperative).  A fixed rule of the launch shape, never a timing,
// so one problem always runs the same arithmetic (the cooperative form sums
// a sample's cost terms in its own order).  MPPI_B200_COOP=1 / 0 pins it on
// (every shape) or off.
bool use_coop(const mppi_backend* b, uint32_t N) {
  if (b->ragged || !b->mod || b->mod->coop_lanes == 0 || N == 0 || b->coop_pin < 0) return false;
  if (b->coop_pin > 0) return true;
  const size_t plain_ctas = (size_t)N * ((b->K + 127) / 128);
  return plain_ctas <= (size_t)b->num_sms / 4;
}

LaunchGeom choose_geometry(const mppi_backend* b, uint32_t N) {
  LaunchGeom g;
  const size_t HM = b->HM();
  const size_t budget = std::min<size_t>(b->max_smem_optin ? b->max_smem_optin : 232448, 232448);
  if (use_coop(b, N)) {
    // 32 samples per CTA (32 * lanes threads) where the one-thread form
    // would have at most one 128-sample CTA per four SMs, so an agent's
    // samples spread over four times as many SMs; otherwise 128 samples
    // (128 * lanes threads, one CTA per SM).  The whole horizon is staged
    // when it fits the SM's shared memory, else in chunks.
    g.coop = b->mod->coop_lanes;
    const size_t plain_ctas = (size_t)N * ((b->K + 127) / 128);
    g.coop_v = plain_ctas <= (size_t)b->num_sms / 4 ? 0 : 1;
    g.block = g.coop_v == 0 ? 32 : 128;
    g.variant = 1;
    const size_t el = b->stage_elem;
    const size_t overhead = b->smem_reserved + b->mod->coop_static_smem[g.coop_v];
    const size_t per_cta =
        std::min(budget, b->smem_per_sm > overhead ? b->smem_per_sm - overhead : (size_t)4096);
    const size_t fixed = nominal_bytes(b) + (size_t)g.block * 4;
    const size_t full = fixed + HM * g.block * el;
    if (full <= per_cta) {
      g.stage_rows = (uint32_t)HM;
      g.smem = full;
    } else {
      uint32_t rows = (uint32_t)((per_cta > fixed ? per_cta - fixed : 0) / ((size_t)g.block * el));
      rows = std::min<uint32_t>(std::max<uint32_t>(b->m, rows / b->m * b->m), (uint32_t)HM);
      g.stage_rows = rows;
      g.smem = fixed + (size_t)rows * g.block * el;
    }
    g.nblk = (b->K + g.block - 1) / g.block;
    g.pstride = (uint32_t)pad4(MPPI_PARTIAL_HEAD + HM);
    return g;
  }
  // Prefer 128 threads; fall back to 64 for very long horizons.
  const int order[2] = {1, 0};
  const size_t el = b->stage_elem;
  // Four 128-thread CTAs per SM (16 warps) hide this kernel's dependency
  // latencies; staging the whole horizon is used only while it keeps that
  // residency, otherwise the noise is staged (and regenerated) in chunks that
  // fill the same per-CTA share of shared memory (the SM's shared memory /
  // 4, less what the system reserves per CTA and the kernel's static part).
  for (int vi : order) {
    const uint32_t block = mppi_b200::kRolloutBlocks[vi];
    const size_t per_cta = rollout_dynamic_share(b, b->mod->rollout_static_smem[vi], budget);
    const size_t fixed = nominal_bytes(b) + (size_t)block * 4;
    const size_t full = fixed + HM * block * el;
    g.variant = vi;
    g.block = block;
    if (full <= per_cta) {
      g.stage_rows = (uint32_t)HM;
      g.smem = full;
      break;
    }
    // A launch whose CTAs are all resident at once with the whole horizon
    // staged (few agents x few samples: one partial wave) gains nothing from
    // the fourth CTA per SM, and chunked staging would regenerate every
    // noise value after the costs are known: stage the whole horizon.
    if (full <= budget && N > 0) {
      const size_t per_sm = b->smem_reserved + b->mod->rollout_static_smem[vi] + full;
      const size_t fit = std::min<size_t>(512 / block, b->smem_per_sm / per_sm);
      const size_t ctas = (size_t)N * ((b->K + block - 1) / block);
      if (fit >= 1 && ctas <= fit * (size_t)b->num_sms) {
        g.stage_rows = (uint32_t)HM;
        g.smem = full;
        break;
      }
    }
    const size_t room = per_cta > fixed + (size_t)block * el * b->m ? per_cta - fixed
                                                                     : (size_t)block * el * b->m;
    uint32_t rows = (uint32_t)(room / ((size_t)block * el));
    rows = std::max<uint32_t>(b->m, rows / b->m * b->m);
    rows = std::min<uint32_t>(rows, (uint32_t)HM);
    g.stage_rows = rows;
    g.smem = fixed + (size_t)rows * block * el;
    if (vi == 1) break;
  }
  g.nblk = (b->K + g.block - 1) / g.block;
  g.pstride = (uint32_t)pad4(MPPI_PARTIAL_HEAD + HM);
  return g;
}

// The geometry of the prepared batch (b->N agents).
LaunchGeom choose_geometry(const mppi_backend* b) { return choose_geometry(b, b->N); }

size_t combine_smem(const mppi_backend* b);

// Dynamic shared memory limit of the current rollout kernels (plain and
// fused forms) for the prepared geometry.
cudaError_t set_rollout_smem(const mppi_backend* b) {
  if (b->geom.smem <= 48 * 1024) return cudaSuccess;
  const void* k[2] = {b->ragged ? (const void*)b->mod->rollout_work
                                : (const void*)b->mod->rollout[b->geom.variant],
                      b->ragged ? (const void*)b->mod->rollout_work_fused
                                : (const void*)b->mod->rollout_fused[b->geom.variant]};
  for (const void* f : k) {
    cudaError_t e =
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->geom.smem);
    if (e != cudaSuccess) return e;
  }
  if (b->geom.coop) {
    for (const void* f :
         {(const void*)b->mod->rollout_coop[b->geom.coop_v],
          (const void*)b->mod->rollout_coop_fused[b->geom.coop_v]}) {
      cudaError_t e =
          cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->geom.smem);
      if (e != cudaSuccess) return e;
    }
  }
  if (!b->ragged) {
    for (const void* f : {(const void*)b->mod->rollout_ws, (const void*)b->mod->rollout_ws_fused,
                          (const void*)b->mod->rollout_early,
                          (const void*)b->mod->rollout_early_fused}) {
      cudaError_t e =
          cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->geom.smem);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

int ensure_shape(mppi_backend* b, uint32_t N, uint32_t T, bool ws, bool wc, bool wk, bool wt,
                 char* err, size_t err_len) {
  bool grew = false;
  CK(cudaStreamSynchronize(b->stream));  // buffers below may be in use
  // the same uniform shape as the previous call (a control loop of steps):
  // buffers and geometry stand
  char key[160];
  snprintf(key, sizeof(key), "%u/%u/%d%d%d%d/%d/%p/%u/%p", N, T, ws, wc, wk, wt, b->record_ustar,
           (const void*)b->proposal, b->prop_samples, (const void*)b->mod.get());
  if (!b->ragged && b->N == N && b->T == T && b->shape_key == key) return MPPI_OK;
  b->shape_key.clear();
  b->N = N;
  b->T = T;
  b->geom = choose_geometry(b);
  if (b->ragged) {
    // uneven batches: 128-thread CTAs (results independent of tuning)
    LaunchGeom g = b->geom;
    if (g.block != 128) {
      const size_t HM = b->HM();
      g.variant = 1;
      g.block = 128;
      uint32_t rows = (uint32_t)(32768 / (128 * b->stage_elem));
      rows = std::min<uint32_t>(std::max<uint32_t>(b->m, rows / b->m * b->m), (uint32_t)HM);
      g.stage_rows = rows;
      g.smem = nominal_bytes(b) + (size_t)128 * 4 + (size_t)rows * 128 * b->stage_elem;
      g.pstride = (uint32_t)pad4(MPPI_PARTIAL_HEAD + HM);
    }
    uint32_t maxblk = 0;
    for (uint32_t a = 0; a < N; ++a) maxblk = std::max(maxblk, (b->agent_K[a] + 127) / 128);
    g.nblk = maxblk;  // the largest agent's CTA count (combine shared memory)
    b->geom = g;
  }
  {
    // zeroed when (re)allocated: the step-form timing of a new shape may run
    // before the first upload, and then reads zeros, not leftover bits
    bool fresh = false;
    CK(b->d_io.ensure(b->io_floats() * 4, &fresh));
    if (fresh) {
      grew = true;
      CK(cudaMemsetAsync(b->d_io.p, 0, b->d_io.bytes, b->stream));
    }
  }
  // per-sample cost pairs, kept by single control steps for inspection
  if (T == 0) CK(b->d_costs.ensure((size_t)2 * N * b->K * 4, &grew));
  const size_t records = b->ragged ? b->total_records : (size_t)N * b->geom.nblk;
  CK(b->d_partials.ensure(records * b->geom.pstride * 4, &grew));
  {
    // the fused combine's counters start at zero (the kernel leaves them so)
    bool fresh = false;
    CK(b->d_done.ensure((size_t)N * 4, &fresh));
    if (fresh) {
      grew = true;
      CK(cudaMemsetAsync(b->d_done.p, 0, b->d_done.bytes, b->stream));
    }
  }
  b->want_s = ws;
  b->want_c = wc;
  b->want_k = wk;
  b->want_t = wt;
  if (ws) CK(b->d_hs.ensure((size_t)T * N * b->n * 4, &grew));
  if (wc) CK(b->d_hc.ensure((size_t)T * N * b->m * 4, &grew));
  if (wk) CK(b->d_hk.ensure((size_t)T * N * 4, &grew));
  if (wt) CK(b->d_term.ensure((size_t)N * b->n * 4, &grew));
  if (b->record_ustar && T) CK(b->d_hu.ensure((size_t)T * N * b->HM() * 4, &grew));
  if (b->proposal) {
    const mppi_b200::ProposalShape ps = mppi_b200::proposal_shape(b->proposal);
    CK(b->d_feat.ensure((size_t)N * kFeatureStride * 4, &grew));
    CK(b->d_prop.ensure((size_t)N * ps.out_stride * 4, &grew));
  }
  CK(b->h_up.ensure((b->off_uout() + 64) * 4 + 2 * pad16(b->mp_size + b->cp_size) + 64));
  CK(b->h_down.ensure((b->io_floats() + 64) * 4));
  if (grew) ++b->generation;
  b->geom.smem = std::max(b->geom.smem, combine_smem(b));  // the fused combine reuses it
  CK(set_rollout_smem(b));
  if (!b->ragged) b->shape_key = key;
  return MPPI_OK;
}

// Whether the attached proposal network runs per agent (inside the combines,
// and for a loop's first step in the rows kernel) rather than as the
// tensor-core batch kernel.  A rule of the batch size, not a timing.
bool net_per_agent(const mppi_backend* b) {
  if (!b->proposal || !b->spec.proposal || b->net_pin < 0 || !b->mod->proposal_rows)
    return false;
  return b->net_pin > 0 || b->N <= kNetPerAgentMax;
}

MppiNetRows net_rows(const mppi_backend* b) {
  MppiNetRows r{};
  const mppi_b200::ProposalWeights w = mppi_b200::proposal_weights(b->proposal);
  for (int l = 0; l < 4; ++l) {
    r.w[l] = w.w[l];
    r.b[l] = w.b[l];
  }
  r.in = w.in;
  r.hidden = w.hidden;
  r.out = w.out;
  r.out_stride = mppi_b200::proposal_shape(b->proposal).out_stride;
  r.out_buf = b->d_prop.as<float>();
  return r;
}

MppiRolloutArgs rollout_args(const mppi_backend* b, uint32_t step_local) {
  MppiRolloutArgs a{};
  a.num_agents = b->N;
  a.K = b->K;
  a.H = b->H;
  a.nblk = b->geom.nblk;
  a.stage_rows = b->geom.stage_rows;
  a.seed = b->seed;
  a.step_local = step_local;
  a.pstride = b->geom.pstride;
  a.lambda = b->lambda;
  a.sigma_stride = b->run_sigma_stride;
  a.sigma_inv_stride = 0;
  a.step_base = reinterpret_cast<const uint32_t*>(b->io());
  a.x = b->io() + b->off_x();
  a.u_nom = b->io() + b->off_unom();
  a.sigma = b->run_sigma;
  a.sigma_inv = b->c_sigma_inv();
  a.u_min = b->c_umin();
  a.u_max = b->c_umax();
  a.model_params = b->run_mp;
  a.cost_params = b->run_cp;
  a.model_stride = b->run_mp_stride;
  a.cost_stride = b->run_cp_stride;
  if (b->T == 0) {  // a single control step: keep its costs for inspection
    a.costs = b->d_costs.as<float>();
    a.costs_lo = a.costs + (size_t)b->N * b->K;
  }
  a.partials = b->d_partials.as<float>();
  if (b->ragged) {
    const uint32_t* info = b->d_agent_info.as<uint32_t>();
    a.agent_K = info;
    a.agent_H = info + b->N;
    a.agent_blk0 = info + 2 * b->N;
    a.work = b->d_work.as<uint2>();
    a.work_counter = b->grid ? b->d_queue.as<uint32_t>() : nullptr;
    a.num_work = b->num_work;
  }
  if (b->proposal && b->spec.proposal) {
    const mppi_b200::ProposalShape ps = mppi_b200::proposal_shape(b->proposal);
    a.prop_out = b->d_prop.as<float>();
    a.prop_stride = ps.out_stride;
    a.prop_count = std::min(b->prop_samples, b->K);
    a.prop_ls_offset = ps.horizon * ps.control_dim;
    a.prop_ls_min = ps.log_scale_min;
    a.prop_ls_max = ps.log_scale_max;
  }
  return a;
}

MppiCombineArgs combine_args(const mppi_backend* b, uint32_t step_local, bool propagate) {
  MppiCombineArgs c{};
  c.num_agents = b->N;
  c.K = b->K;
  c.H = b->H;
  c.nblk = b->geom.nblk;
  c.pstride = b->geom.pstride;
  c.step_local = step_local;
  c.lambda = b->lambda;
  c.propagate = propagate ? 1u : 0u;
  c.step_base = reinterpret_cast<const uint32_t*>(b->io());
  c.partials = b->d_partials.as<float>();
  c.u_min = b->c_umin();
  c.u_max = b->c_umax();
  c.model_params = b->run_mp;
  c.model_stride = b->run_mp_stride;
  c.u_nom = b->io() + b->off_unom();
  c.u_out = b->io() + b->off_uout();
  c.diag = b->io() + b->off_diag();
  c.stats = b->io() + b->off_stats();
  c.x = b->io() + b->off_x();
  c.hist_states = b->want_s ? b->d_hs.as<float>() : nullptr;
  c.hist_controls = b->want_c ? b->d_hc.as<float>() : nullptr;
  c.hist_costs = b->want_k ? b->d_hk.as<float>() : nullptr;
  c.terminal = b->want_t ? b->d_term.as<float>() : nullptr;
  c.hist_ustar = (b->record_ustar && b->T > 0 && propagate) ? b->d_hu.as<float>() : nullptr;
  if (propagate && b->proposal && b->spec.proposal) {
    // features of the propagated state feed the next step's network
    c.cost_params = b->run_cp;
    c.cost_stride = b->run_cp_stride;
    c.features = b->d_feat.as<float>();
    c.feature_stride = kFeatureStride;
    // the next step's network output by the combine's threads
    if (net_per_agent(b)) c.net = net_rows(b);
  }
  if (b->ragged) {
    const uint32_t* info = b->d_agent_info.as<uint32_t>();
    c.agent_K = info;
    c.agent_H = info + b->N;
    c.agent_blk0 = info + 2 * b->N;
    c.block = 128;
  }
  return c;
}

size_t combine_smem(const mppi_backend* b) {
  return (pad4(b->geom.nblk) + pad4(b->HM())) * 4;
}

// Proposal features of the current states (the closed loop computes them
// inside the previous step's combine instead, once it has the new state).
cudaError_t launch_features(mppi_backend* b) {
  MppiFeaturesArgs f{};
  f.rows = b->N;
  f.agents_mod = b->N;
  f.x_stride = b->n;
  f.out_stride = kFeatureStride;
  f.x = b->io() + b->off_x();
  f.model_params = b->run_mp;
  f.cost_params = b->run_cp;
  f.model_stride = b->run_mp_stride;
  f.cost_stride = b->run_cp_stride;
  f.out = b->d_feat.as<float>();
  void* fa[] = {&f};
  return cudaLaunchKernel((const void*)b->mod->features, dim3((b->N + 127) / 128), dim3(128), fa,
                          0, b->stream);
}

// The network's forward pass on the current features.
cudaError_t launch_network(mppi_backend* b) {
  return mppi_b200::proposal_enqueue_forward(b->proposal, b->stream, b->d_feat.as<float>(),
                                             kFeatureStride, b->N, b->d_prop.as<float>(),
                                             b->pdl);
}

// Features and the network per agent, one CTA per agent (the rows kernel);
// given_features: the network alone on the features already in d_feat.
cudaError_t launch_proposal_rows(mppi_backend* b, bool given_features = false) {
  MppiProposalRowsArgs a{};
  a.given_features = given_features ? 1u : 0u;
  a.f.rows = b->N;
  a.f.agents_mod = b->N;
  a.f.x_stride = b->n;
  a.f.out_stride = kFeatureStride;
  a.f.x = b->io() + b->off_x();
  a.f.model_params = b->run_mp;
  a.f.cost_params = b->run_cp;
  a.f.model_stride = b->run_mp_stride;
  a.f.cost_stride = b->run_cp_stride;
  a.f.out = b->d_feat.as<float>();
  a.net = net_rows(b);
  void* args[] = {&a};
  return cudaLaunchKernel((const void*)b->mod->proposal_rows, dim3(b->N), dim3(128), args, 0,
                          b->stream);
}

// Features, then the network (both on the backend stream): per agent in one
// kernel, or the features kernel and the tensor-core batch kernel.
cudaError_t launch_proposal(mppi_backend* b) {
  if (net_per_agent(b)) return launch_proposal_rows(b);
  cudaError_t e = launch_features(b);
  return e == cudaSuccess ? launch_network(b) : e;
}

// A launch on the backend stream that may start while the previous kernel
// finishes (programmatic stream serialisation): the kernel's CTAs run their
// loop-constant prologue and then wait (griddepcontrol.wait) for the
// previous grid to complete before they read anything it writes.
cudaError_t launch_dependent(const mppi_backend* b, const void* func, dim3 grid, dim3 block,
                             size_t smem, void** args) {
  if (!b->pdl) return cudaLaunchKernel(func, grid, block, args, smem, b->stream);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = b->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, func, args);
}

// The one-thread 128-sample form with the early noise (drawn before the
// wait for the previous launch): uniform batches with the whole horizon
// staged and no proposal attached.  Same bits as mppi_rollout_b128; its own
// entry, because the early path's extra live state cost the chunked
// quadrotor rollout 132 bytes of spills.
bool early_noise(const mppi_backend* b) {
  return !b->no_early && !b->ragged && !b->geom.coop && b->geom.variant == 1 &&
         b->geom.block == 128 && b->geom.stage_rows >= b->HM() &&
         !(b->proposal && b->spec.proposal);
}

// A rollout launch with prepared arguments (uniform grid, or the uneven
// batch's work items).
cudaError_t launch_rollout_args(mppi_backend* b, MppiRolloutArgs& a, bool ws = false) {
  void* args[] = {&a};
  const bool fused = a.agent_done != nullptr;
  if (ws && !b->ragged)
    return launch_dependent(b, fused ? (const void*)b->mod->rollout_ws_fused
                                     : (const void*)b->mod->rollout_ws,
                            dim3(b->geom.nblk, b->N), dim3(2 * b->geom.block), b->geom.smem,
                            args);
  if (b->ragged) {
    const void* f = fused ? (const void*)b->mod->rollout_work_fused
                          : (const void*)b->mod->rollout_work;
    // one CTA per work item: a dependent launch like the uniform batch's;
    // a persistent grid's queue counter is reset first (a plain launch)
    if (!b->grid) return launch_dependent(b, f, dim3(b->num_work), dim3(128), b->geom.smem, args);
    cudaError_t e = cudaMemsetAsync(b->d_queue.p, 0, 4, b->stream);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernel(f, dim3(b->grid), dim3(128), args, b->geom.smem, b->stream);
  }
  if (b->geom.coop)
    return launch_dependent(b, fused ? (const void*)b->mod->rollout_coop_fused[b->geom.coop_v]
                                     : (const void*)b->mod->rollout_coop[b->geom.coop_v],
                            dim3(b->geom.nblk, b->N), dim3(b->geom.block * b->geom.coop),
                            b->geom.smem, args);
  if (early_noise(b))
    return launch_dependent(b, fused ? (const void*)b->mod->rollout_early_fused
                                     : (const void*)b->mod->rollout_early,
                            dim3(b->geom.nblk, b->N), dim3(b->geom.block), b->geom.smem, args);
  return launch_dependent(b, fused ? (const void*)b->mod->rollout_fused[b->geom.variant]
                                   : (const void*)b->mod->rollout[b->geom.variant],
                          dim3(b->geom.nblk, b->N), dim3(b->geom.block), b->geom.smem, args);
}

// The rollout kernel alone (the proposal's outputs already in place).
cudaError_t launch_rollout_kernel(mppi_backend* b, uint32_t step_local) {
  MppiRolloutArgs a = rollout_args(b, step_local);
  return launch_rollout_args(b, a);
}

// One rollout pass: the proposal's features and network first when one is
// attached, then the rollout kernel.
cudaError_t launch_rollout(mppi_backend* b, uint32_t step_local) {
  if (b->proposal && b->spec.proposal) {
    cudaError_t e = launch_proposal(b);
    if (e != cudaSuccess) return e;
  }
  return launch_rollout_kernel(b, step_local);
}

// Uneven batches: times candidate (grid size, noise staging) pairs on the
// prepared data and keeps the fastest.  Every candidate computes the same
// bits (same 128-thread partition of samples, same summation orders).
int tune_ragged(mppi_backend* b, char* err, size_t err_len) {
  const size_t HM = b->HM();
  const size_t budget = std::min<size_t>(b->max_smem_optin ? b->max_smem_optin : 232448, 232448);
  std::vector<uint32_t> stage_options;
  const size_t el = b->stage_elem;
  const size_t full = nominal_bytes(b) + 128 * 4 + HM * 128 * el;
  if (full <= budget - 2048) stage_options.push_back((uint32_t)HM);
  uint32_t chunk = std::max<uint32_t>(b->m, (uint32_t)(32768 / (128 * el)) / b->m * b->m);
  stage_options.push_back(std::min<uint32_t>(chunk, (uint32_t)HM));
  std::vector<uint32_t> grids = {0};
  for (uint32_t c = 1; c <= 4; ++c) grids.push_back(c * (uint32_t)b->num_sms);
  // MPPI_B200_UNEVEN_GRID / MPPI_B200_UNEVEN_STAGE_ROWS pin a candidate
  // (reproducible profiling; the result bits are the same either way)
  if (const char* g = getenv("MPPI_B200_UNEVEN_GRID"); g && *g) {
    grids.assign(1, (uint32_t)strtoul(g, nullptr, 10));
  }
  if (const char* r = getenv("MPPI_B200_UNEVEN_STAGE_ROWS"); r && *r) {
    const uint32_t rows = (uint32_t)strtoul(r, nullptr, 10);
    if (rows >= b->m && rows % b->m == 0) {
      const size_t sm = nominal_bytes(b) + 128 * 4 + (size_t)std::min<size_t>(rows, HM) * 128 * el;
      if (sm <= budget) stage_options.assign(1, (uint32_t)std::min<size_t>(rows, HM));
    }
  }
  const LaunchGeom base = b->geom;
  float best = 1e30f;
  LaunchGeom best_g = base;
  uint32_t best_grid = 0;
  for (uint32_t rows : stage_options) {
    LaunchGeom g = base;
    g.stage_rows = rows;
    g.smem = std::max(nominal_bytes(b) + 128 * 4 + (size_t)rows * 128 * el, combine_smem(b));
    b->geom = g;
    CK(cudaFuncSetAttribute((const void*)b->mod->rollout_work,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem));
    for (uint32_t grid : grids) {
      b->grid = grid;
      CK(launch_rollout(b, 0));  // warm-up
      CK(cudaEventRecord(b->ev0, b->stream));
      for (int i = 0; i < 3; ++i) CK(launch_rollout(b, 0));
      CK(cudaEventRecord(b->ev1, b->stream));
      CK(cudaEventSynchronize(b->ev1));
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
      ms /= 3.0f;
      if (ms < best) {
        best = ms;
        best_g = g;
        best_grid = grid;
      }
    }
  }
  b->geom = best_g;
  b->grid = best_grid;
  b->tuned_ms = best;
  b->tuned_geom = best_g;
  b->tuned_grid = best_grid;
  CK(cudaFuncSetAttribute((const void*)b->mod->rollout_work,
                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)best_g.smem));
  CK(set_rollout_smem(b));
  return MPPI_OK;
}

std::string ragged_key(const mppi_backend* b) {
  std::string k = std::to_string(b->N) + ":";
  for (uint32_t a = 0; a < b->N; ++a)
    k += std::to_string(b->agent_K[a]) + "," + std::to_string(b->agent_H[a]) + ";";
  return k;
}

cudaError_t launch_combine(mppi_backend* b, uint32_t step_local, bool propagate) {
  MppiCombineArgs c = combine_args(b, step_local, propagate);
  void* args[] = {&c};
  return cudaLaunchKernel((const void*)b->mod->combine, dim3(b->N), dim3(256), args,
                          combine_smem(b), b->stream);
}

constexpr uint32_t kFormFused = 1;  // combine run by each agent's last rollout CTA
constexpr uint32_t kFormWs = 2;     // warp-specialised rollout (noise drawn by extra warps)

bool fused_combine(const mppi_backend* b) { return (b->form & kFormFused) != 0; }

// The warp-specialised rollout needs 128-sample CTAs with the whole horizon
// staged, in a uniform batch.
bool ws_possible(const mppi_backend* b) {
  return !b->ragged && !b->geom.coop && b->geom.block == 128 && b->geom.stage_rows >= b->HM();
}

// One step's kernels after the proposal stage in the given form: the rollout
// (plain or warp-specialised) with the combine run by each agent's last CTA,
// or the rollout and combine kernels.
cudaError_t launch_step_form(mppi_backend* b, uint32_t step_local, bool propagate,
                             uint32_t form) {
  MppiRolloutArgs a = rollout_args(b, step_local);
  if (form & kFormFused) {
    a.agent_done = b->d_done.as<uint32_t>();
    a.comb = combine_args(b, step_local, propagate);
    return launch_rollout_args(b, a, (form & kFormWs) != 0);
  }
  cudaError_t e = launch_rollout_args(b, a, (form & kFormWs) != 0);
  return e == cudaSuccess ? launch_combine(b, step_local, propagate) : e;
}

cudaError_t launch_rollout_combine(mppi_backend* b, uint32_t step_local, bool propagate) {
  return launch_step_form(b, step_local, propagate, b->form);
}

// Chooses the form of a step for the prepared launch shape -- combine fused
// into the rollout or not, warp-specialised rollout or not -- by timing the
// candidates (after a warm-up, three steps each, the proposal stage first
// when a network is attached, as in the loop; without propagation, so no
// state changes), once per shape, as the uneven-batch tuner does.  Every form
// computes the same bits.  The fused combine saves a launch but its tail can
// cost a model's rollout registers; the warp-specialised rollout shortens
// each sample's chain where few CTAs leave SMs idle, and only costs
// instructions where the SMs are full -- so neither choice wins everywhere.
int decide_step_form(mppi_backend* b, char* err, size_t err_len) {
  char kb[192];
  snprintf(kb, sizeof(kb), "%u/%u/%u/%d/%u/%u/%u/%u/%p/%p/%u/%d/", b->N, b->K, b->H,
           b->geom.variant, b->geom.block, b->geom.stage_rows, b->geom.nblk, b->grid,
           (const void*)b->mod.get(), (const void*)b->proposal, b->prop_samples, (int)b->ragged);
  const std::string key = std::string(kb) + (b->ragged ? b->tuned_key : std::string());
  if (b->form_key == key) return MPPI_OK;
  std::vector<uint32_t> forms;
  for (uint32_t ws : {0u, kFormWs}) {
    if (ws && (b->ws_pin < 0 || !ws_possible(b))) continue;
    if (!ws && b->ws_pin > 0 && ws_possible(b)) continue;
    for (uint32_t fu : {0u, kFormFused}) {
      if (fu && b->combine_pin < 0) continue;
      if (!fu && b->combine_pin > 0) continue;
      forms.push_back(ws | fu);
    }
  }
  uint32_t best = forms.front();
  if (forms.size() > 1) {
    CK(set_rollout_smem(b));
    float best_ms = 1e30f;
    for (int pass = 0; pass < 2; ++pass) {
      for (uint32_t f : forms) {
        const int reps = pass ? 3 : 1;
        CK(cudaEventRecord(b->ev0, b->stream));
        for (int i = 0; i < reps; ++i) {
          if (b->proposal && b->spec.proposal) CK(launch_proposal(b));
          CK(launch_step_form(b, 0, false, f));
        }
        CK(cudaEventRecord(b->ev1, b->stream));
        CK(cudaEventSynchronize(b->ev1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        if (pass && ms < best_ms) {
          best_ms = ms;
          best = f;
        }
      }
    }
  }
  b->form = best;
  b->form_key = key;
  return MPPI_OK;
}

// Resolves the parameter blob pointers of a run: per-agent blobs, an
// override, the bound blob, or a zero word (the reference binds a 1-byte zero
// buffer when nothing is bound, metal_backend.mm:595-600).
const uint8_t* pick_params(mppi_backend* b, bool is_model, const void* ovr, size_t ovr_bytes) {
  DevBuf& bound = is_model ? b->d_mp_bound : b->d_cp_bound;
  DevBuf& obuf = is_model ? b->d_mp_ovr : b->d_cp_ovr;
  const bool has_bound = is_model ? b->mp_bound : b->cp_bound;
  if (ovr != nullptr && ovr_bytes > 0) return obuf.as<uint8_t>();
  if (has_bound) return bound.as<uint8_t>();
  return b->d_zero.as<uint8_t>();
}

int check_init(mppi_backend* b, char* err, size_t err_len) {
  if (b == nullptr) {
    set_err(err, err_len, "backend handle is null.");
    return MPPI_ERR_INVALID;
  }
  if (!b->initialized) {
    set_err(err, err_len, "MPPI backend is not initialized.");
    return MPPI_ERR_NOT_INIT;
  }
  cudaError_t e = cudaSetDevice(b->device);
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("cudaSetDevice failed: ") + cudaGetErrorString(e));
    return MPPI_ERR_CUDA;
  }
  return MPPI_OK;
}

// Stages [step_base][x][u_nom] (and blob overrides) in the pinned upload
// buffer; issue_upload then copies them with one transfer each.  The
// caller has synchronised the stream (the buffer may still feed a copy).
void stage_upload(mppi_backend* b, uint64_t start_step, const float* x, const float* u_nom,
                  const void* mp_ovr, size_t mp_bytes, const void* cp_ovr, size_t cp_bytes) {
  float* up = b->h_up.as<float>();
  const size_t nx = (size_t)b->N * b->n, nu = (size_t)b->N * b->HM();
  uint32_t sb = (uint32_t)start_step;
  memcpy(up, &sb, 4);
  memcpy(up + b->off_x(), x, nx * 4);
  if (u_nom)
    memcpy(up + b->off_unom(), u_nom, nu * 4);
  else
    memset(up + b->off_unom(), 0, nu * 4);
  uint8_t* tail = reinterpret_cast<uint8_t*>(up + b->off_uout());
  if (mp_ovr && mp_bytes) {
    memset(tail, 0, pad16(b->mp_size));
    memcpy(tail, mp_ovr, mp_bytes);
    tail += pad16(b->mp_size);
  }
  if (cp_ovr && cp_bytes) {
    memset(tail, 0, pad16(b->cp_size));
    memcpy(tail, cp_ovr, cp_bytes);
  }
}

cudaError_t issue_upload(mppi_backend* b, bool mp_ovr, bool cp_ovr) {
  float* up = b->h_up.as<float>();
  cudaError_t e =
      cudaMemcpyAsync(b->io(), up, b->off_uout() * 4, cudaMemcpyHostToDevice, b->stream);
  uint8_t* tail = reinterpret_cast<uint8_t*>(up + b->off_uout());
  if (e == cudaSuccess && mp_ovr) {
    e = cudaMemcpyAsync(b->d_mp_ovr.p, tail, pad16(b->mp_size), cudaMemcpyHostToDevice,
                        b->stream);
    tail += pad16(b->mp_size);
  }
  if (e == cudaSuccess && cp_ovr)
    e = cudaMemcpyAsync(b->d_cp_ovr.p, tail, pad16(b->cp_size), cudaMemcpyHostToDevice,
                        b->stream);
  return e;
}

// Uploads [step_base][x][u_nom] (and blob overrides) with one pinned copy each.
int upload_state(mppi_backend* b, uint64_t start_step, const float* x, const float* u_nom,
                 const void* mp_ovr, size_t mp_bytes, const void* cp_ovr, size_t cp_bytes,
                 char* err, size_t err_len) {
  // the pinned staging buffer may still feed an earlier asynchronous copy
  CK(cudaStreamSynchronize(b->stream));
  const bool mo = mp_ovr && mp_bytes, co = cp_ovr && cp_bytes;
  if (mo) CK(b->d_mp_ovr.ensure(pad16(b->mp_size)));
  if (co) CK(b->d_cp_ovr.ensure(pad16(b->cp_size)));
  stage_upload(b, start_step, x, u_nom, mp_ovr, mp_bytes, cp_ovr, cp_bytes);
  CK(issue_upload(b, mo, co));
  return MPPI_OK;
}

int check_override_sizes(mppi_backend* b, size_t mp_bytes, const void* mp, size_t cp_bytes,
                         const void* cp, char* err, size_t err_len) {
  if (mp && mp_bytes > 0 && mp_bytes != b->mp_size) {
    set_err(err, err_len,
            "model_params_override.bytes (" + std::to_string(mp_bytes) +
                ") does not match ParamLayout::model_params_size (" +
                std::to_string(b->mp_size) + ").");
    return MPPI_ERR_INVALID;
  }
  if (cp && cp_bytes > 0 && cp_bytes != b->cp_size) {
    set_err(err, err_len,
            "cost_params_override.bytes (" + std::to_string(cp_bytes) +
                ") does not match ParamLayout::cost_params_size (" +
                std::to_string(b->cp_size) + ").");
    return MPPI_ERR_INVALID;
  }
  return MPPI_OK;
}

// Enqueues T closed-loop steps (rollout with combine/propagate each), through a
// CUDA graph captured once per (shape, buffers) and replayed afterwards.
int enqueue_closed_loop(mppi_backend* b, char* err, size_t err_len) {
  char keybuf[320];
  snprintf(keybuf, sizeof(keybuf), "%u/%u/%llu/%d/%d%d%d%d%d/%p/%p/%llu/%llu/%p/%u/%p/%u/%p",
           b->N, b->T, (unsigned long long)b->generation, b->geom.variant, b->want_s, b->want_c,
           b->want_k, b->want_t, b->record_ustar, (const void*)b->run_mp, (const void*)b->run_cp,
           (unsigned long long)b->run_mp_stride, (unsigned long long)b->run_cp_stride,
           (const void*)b->run_sigma, b->run_sigma_stride, (const void*)b->proposal,
           b->prop_samples, (const void*)b->mod.get());
  if (b->ragged) {
    const std::string rk = ragged_key(b);
    if (b->tuned_key != rk) {
      if (int rc = tune_ragged(b, err, err_len)) return rc;
      b->tuned_key = rk;
    } else {
      // prepare() re-derived the default geometry; restore the tuned one
      b->geom = b->tuned_geom;
      b->grid = b->tuned_grid;
      CK(set_rollout_smem(b));
    }
  }
  if (int rc = decide_step_form(b, err, err_len)) return rc;
  const std::string key = std::string(keybuf) + (b->ragged ? "/r" + std::to_string(b->grid) + "/" +
                                                                 std::to_string(b->geom.stage_rows) +
                                                                 "/" + b->tuned_key
                                                           : std::string()) +
                          "/form" + std::to_string(b->form);
  if (b->graph == nullptr || b->graph_key != key) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = cudaSuccess;
    const bool prop = b->proposal && b->spec.proposal;
    // with a proposal: features of x0 once, then per step network -> rollout
    // -> combine (which leaves the next step's features behind); with the
    // per-agent network the first step's kernel evaluates it for x0 and each
    // combine evaluates it for the next step
    const bool per_agent = prop && net_per_agent(b);
    if (prop) le = per_agent ? launch_proposal_rows(b) : launch_features(b);
    for (uint32_t s = 0; s < b->T && le == cudaSuccess; ++s) {
      if (prop && !per_agent) le = launch_network(b);
      if (le == cudaSuccess) le = launch_rollout_combine(b, s, true);
    }
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      set_err(err, err_len, std::string("graph capture failed: ") +
                                cudaGetErrorString(le != cudaSuccess ? le : ce));
      return MPPI_ERR_CUDA;
    }
    cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    b->graph_key = key;
  }
  CK(cudaGraphLaunch(b->graph, b->stream));
  return MPPI_OK;
}

// Per-sample costs and weights exist for the last single control step only
// (dispatch_rollout): the closed loops do not write them.
int check_step_costs(mppi_backend* b, uint32_t a0, uint32_t n, const float* out, char* err,
                     size_t err_len) {
  if (b->T != 0 || b->d_costs.p == nullptr) {
    set_err(err, err_len,
            "per-sample costs are kept by dispatch_rollout only (closed loops do not write "
            "them); run a single control step first.");
    return MPPI_ERR_INVALID;
  }
  if (!out || a0 + n > b->N) {
    set_err(err, err_len, "agent range out of bounds.");
    return MPPI_ERR_INVALID;
  }
  return MPPI_OK;
}

}  // namespace

extern "C" {

const char* mppi_b200_version(void) { return "mppi_metal_b200 0.1.0 (sm_100a)"; }

int mppi_backend_create(mppi_backend** out) {
  if (!out) return MPPI_ERR_INVALID;
  *out = new (std::nothrow) mppi_backend();
  if (*out) {
    const char* sep = getenv("MPPI_B200_SEPARATE_COMBINE");
    (*out)->fuse_combine = !(sep && *sep && *sep != '0');
    const char* nopdl = getenv("MPPI_B200_NO_PDL");
    (*out)->pdl = !(nopdl && *nopdl && *nopdl != '0');
    const char* fc = getenv("MPPI_B200_FUSED_COMBINE");
    if (fc && *fc && *fc != '0') (*out)->combine_pin = 1;
    if (!(*out)->fuse_combine) (*out)->combine_pin = -1;
    if (const char* ws = getenv("MPPI_B200_WS"); ws && *ws) (*out)->ws_pin = *ws == '0' ? -1 : 1;
    if (const char* co = getenv("MPPI_B200_COOP"); co && *co)
      (*out)->coop_pin = *co == '0' ? -1 : 1;
    if (const char* np = getenv("MPPI_B200_NET_PER_AGENT"); np && *np)
      (*out)->net_pin = *np == '0' ? -1 : 1;
    if (const char* ne = getenv("MPPI_B200_NO_EARLY_NOISE"); ne && *ne && *ne != '0')
      (*out)->no_early = true;
  }
  return *out ? MPPI_OK : MPPI_ERR_INVALID;
}

void mppi_backend_destroy(mppi_backend* b) {
  if (!b) return;
  if (b->initialized) cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  delete b;
}

int mppi_backend_initialize(mppi_backend* b, const mppi_backend_plugin* plugin,
                            const mppi_backend_config* cfg, char* err, size_t err_len) {
  if (!b || !plugin || !cfg) {
    set_err(err, err_len, "null argument to mppi_backend_initialize.");
    return MPPI_ERR_INVALID;
  }
  if (cfg->state_dim == 0 || cfg->control_dim == 0 || cfg->horizon == 0 ||
      cfg->sample_count == 0) {
    set_err(err, err_len, "state_dim, control_dim, horizon and sample_count must be > 0.");
    return MPPI_ERR_INVALID;
  }
  if (cfg->state_dim > MPPI_MAX_STATE_DIM) {
    set_err(err, err_len, "DriverConfig::state_dim (" + std::to_string(cfg->state_dim) +
                              ") exceeds the state limit of " +
                              std::to_string(MPPI_MAX_STATE_DIM) + " floats.");
    return MPPI_ERR_INVALID;
  }
  if (cfg->control_dim > 16) {
    set_err(err, err_len, "DriverConfig::control_dim (" + std::to_string(cfg->control_dim) +
                              ") exceeds MPPI_MAX_CONTROL_DIM = 16.");
    return MPPI_ERR_INVALID;
  }
  if (!cfg->sigma || !cfg->u_min || !cfg->u_max || (cfg->control_cost && !cfg->sigma_inv)) {
    set_err(err, err_len, "sigma, sigma_inv, u_min and u_max must not be null.");
    return MPPI_ERR_INVALID;
  }
  if (!plugin->source_path || !*plugin->source_path) {
    set_err(err, err_len, "user_metallib_path is empty.");
    return MPPI_ERR_PLUGIN;
  }
  if (!valid_identifier(plugin->dynamics)) {
    set_err(err, err_len, std::string("Required callable '") +
                              (plugin->dynamics ? plugin->dynamics : "") +
                              "' is not a valid identifier.");
    return MPPI_ERR_CALLABLE;
  }
  for (const char* nm : {plugin->stage_cost, plugin->terminal_cost}) {
    if (nm && *nm && !valid_identifier(nm)) {
      set_err(err, err_len, std::string("Callable '") + nm + "' is not a valid identifier.");
      return MPPI_ERR_CALLABLE;
    }
  }

  // ---- device (metal_backend.mm:227-231: the default device) ----
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    set_err(err, err_len, std::string("No CUDA device available: ") +
                              (e != cudaSuccess ? cudaGetErrorString(e) : "device count is 0"));
    return MPPI_ERR_NO_DEVICE;
  }
  CK(cudaGetDevice(&b->device));
  cudaDeviceProp prop{};
  CK(cudaGetDeviceProperties(&prop, b->device));
  if (prop.major < 10) {
    set_err(err, err_len, std::string("device '") + prop.name +
                              "' is not sm_100 (Blackwell); this library is built for sm_100a.");
    return MPPI_ERR_NO_DEVICE;
  }
  b->num_sms = prop.multiProcessorCount;
  b->max_smem_optin = prop.sharedMemPerBlockOptin;
  b->smem_per_sm = prop.sharedMemPerMultiprocessor;
  b->smem_reserved = prop.reservedSharedMemPerBlock;

  b->n = cfg->state_dim;
  b->m = cfg->control_dim;
  b->H = cfg->horizon;
  b->K = cfg->sample_count;
  b->lambda = cfg->lambda;
  b->cov_full = cfg->covariance_form == 1;
  b->control_cost = cfg->control_cost != 0;
  b->noise_half = cfg->numeric_mode != 0;  // kFp16 and kMixed: FP16 noise
  b->stage_elem = b->noise_half ? 2 : 4;
  b->seed = (uint32_t)plugin->seed;  // metal_backend.mm:565
  b->mp_size = plugin->model_params_size;
  b->cp_size = plugin->cost_params_size;
  const uint32_t m = b->m;
  if (b->cov_full) {
    if (!cholesky(m, cfg->sigma, &b->sigma_dev)) {
      set_err(err, err_len, "ControlNoiseConfig::sigma (kFull) is not symmetric positive definite.");
      return MPPI_ERR_INVALID;
    }
  } else {
    b->sigma_dev.assign(cfg->sigma, cfg->sigma + m);
  }
  const size_t sl = b->cov_full ? (size_t)m * m : m;
  if (cfg->sigma_inv)
    b->sigma_inv.assign(cfg->sigma_inv, cfg->sigma_inv + sl);
  else
    b->sigma_inv.assign(sl, 0.0f);
  b->u_min.assign(cfg->u_min, cfg->u_min + m);
  b->u_max.assign(cfg->u_max, cfg->u_max + m);

  // ---- kernel module: plugin + library kernels (metal_backend.mm:278-560) ----
  mppi_b200::ModuleSpec spec;
  spec.plugin_path = plugin->source_path;
  spec.dynamics = plugin->dynamics;
  spec.stage_cost = plugin->stage_cost ? plugin->stage_cost : "";
  spec.terminal_cost = plugin->terminal_cost ? plugin->terminal_cost : "";
  spec.state_dim = b->n;
  spec.control_dim = m;
  spec.cov_full = b->cov_full;
  spec.control_cost = b->control_cost;
  spec.noise_half = b->noise_half;
  spec.model_params_bytes = b->mp_size;
  spec.cost_params_bytes = b->cp_size;
  spec.model_params_alignment = plugin->model_params_alignment ? plugin->model_params_alignment : 1;
  spec.cost_params_alignment = plugin->cost_params_alignment ? plugin->cost_params_alignment : 1;
  spec.schema_hash = plugin->schema_hash ? plugin->schema_hash : "";
  std::string merr;
  const int rc = mppi_b200::load_module(spec, &b->mod, &merr);
  if (rc != MPPI_OK) {
    set_err(err, err_len, merr);
    return rc;
  }
  b->spec = spec;
  b->proposal = nullptr;
  b->feature_dim = 0;

  if (!b->stream) CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  if (!b->ev0) CK(cudaEventCreate(&b->ev0));
  if (!b->ev1) CK(cudaEventCreate(&b->ev1));

  // constants: [sigma (m*m)][sigma_inv (m*m)][u_min][u_max]
  const size_t mm = pad4((size_t)m * m);
  std::vector<float> consts(2 * mm + 2 * pad4(m), 0.0f);
  std::copy(b->sigma_dev.begin(), b->sigma_dev.end(), consts.begin());
  std::copy(b->sigma_inv.begin(), b->sigma_inv.end(), consts.begin() + mm);
  std::copy(b->u_min.begin(), b->u_min.end(), consts.begin() + 2 * mm);
  std::copy(b->u_max.begin(), b->u_max.end(), consts.begin() + 2 * mm + pad4(m));
  CK(b->d_consts.ensure(consts.size() * 4));
  CK(cudaMemcpy(b->d_consts.p, consts.data(), consts.size() * 4, cudaMemcpyHostToDevice));
  CK(b->d_zero.ensure(std::max<size_t>(256, pad16(std::max(b->mp_size, b->cp_size)))));
  CK(cudaMemset(b->d_zero.p, 0, b->d_zero.bytes));
  b->initialized = true;
  return MPPI_OK;
}

int mppi_backend_bind_params(mppi_backend* b, const void* mp, size_t mp_bytes, const void* cp,
                             size_t cp_bytes, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  CK(cudaStreamSynchronize(b->stream));
  if (mp && mp_bytes > 0) {
    if (mp_bytes != b->mp_size) {
      set_err(err, err_len, "model_params.bytes does not match ParamLayout::model_params_size.");
      return MPPI_ERR_INVALID;
    }
    std::vector<uint8_t> tmp(pad16(mp_bytes), 0);
    memcpy(tmp.data(), mp, mp_bytes);
    CK(b->d_mp_bound.ensure(tmp.size()));
    CK(cudaMemcpy(b->d_mp_bound.p, tmp.data(), tmp.size(), cudaMemcpyHostToDevice));
    b->mp_bound = true;
  } else {
    b->mp_bound = false;
  }
  if (cp && cp_bytes > 0) {
    if (cp_bytes != b->cp_size) {
      set_err(err, err_len, "cost_params.bytes does not match ParamLayout::cost_params_size.");
      return MPPI_ERR_INVALID;
    }
    std::vector<uint8_t> tmp(pad16(cp_bytes), 0);
    memcpy(tmp.data(), cp, cp_bytes);
    CK(b->d_cp_bound.ensure(tmp.size()));
    CK(cudaMemcpy(b->d_cp_bound.p, tmp.data(), tmp.size(), cudaMemcpyHostToDevice));
    b->cp_bound = true;
  } else {
    b->cp_bound = false;
  }
  return MPPI_OK;
}

int mppi_backend_dispatch_rollout(mppi_backend* b, uint64_t step_index, const float* x0,
                                  const float* u_nominal, const void* mp, size_t mp_bytes,
                                  const void* cp, size_t cp_bytes, float* u_out, float* diag3,
                                  char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (!x0 || !u_nominal || !u_out) {
    set_err(err, err_len, "x0, u_nominal and u_out must not be null.");
    return MPPI_ERR_INVALID;
  }
  if (int rc = check_override_sizes(b, mp_bytes, mp, cp_bytes, cp, err, err_len)) return rc;
  b->ragged = false;
  if (int rc = ensure_shape(b, 1, 0, false, false, false, false, err, err_len)) return rc;
  b->run_mp = pick_params(b, true, mp, mp_bytes);
  b->run_cp = pick_params(b, false, cp, cp_bytes);
  b->run_mp_stride = b->run_cp_stride = 0;
  b->run_sigma = b->c_sigma();
  b->run_sigma_stride = 0;
  const bool mo = mp && mp_bytes, co = cp && cp_bytes;
  if (mo) CK(b->d_mp_ovr.ensure(pad16(b->mp_size)));
  if (co) CK(b->d_cp_ovr.ensure(pad16(b->cp_size)));
  if (int rc = decide_step_form(b, err, err_len)) return rc;
  stage_upload(b, step_index, x0, u_nominal, mp, mp_bytes, cp, cp_bytes);
  float* down = b->h_down.as<float>();
  const size_t nd = b->off_stats() - b->off_uout();
  // The whole step -- uploads from the pinned staging buffer, the proposal
  // stage if attached, rollout, combine, download -- is one CUDA graph,
  // captured once per (buffers, parameter pointers, module) and replayed:
  // one launch per control step instead of four or five API calls.
  char keybuf[256];
  snprintf(keybuf, sizeof(keybuf), "%u/%llu/%p/%p/%d%d/%p/%u/%p/%p/%p", b->form,
           (unsigned long long)b->generation, (const void*)b->run_mp, (const void*)b->run_cp,
           mo, co, (const void*)b->proposal, b->prop_samples, (const void*)b->mod.get(),
           b->h_up.p, b->h_down.p);
  if (b->step_graph == nullptr || b->step_key != keybuf) {
    if (b->step_graph) {
      cudaGraphExecDestroy(b->step_graph);
      b->step_graph = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t le = issue_upload(b, mo, co);
    if (le == cudaSuccess && b->proposal && b->spec.proposal) le = launch_proposal(b);
    if (le == cudaSuccess) le = launch_rollout_combine(b, 0, false);
    if (le == cudaSuccess)
      le = cudaMemcpyAsync(down, b->io() + b->off_uout(), nd * 4, cudaMemcpyDeviceToHost,
                           b->stream);
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      set_err(err, err_len, std::string("step graph capture failed: ") +
                                cudaGetErrorString(le != cudaSuccess ? le : ce));
      return MPPI_ERR_CUDA;
    }
    cudaError_t ie = cudaGraphInstantiate(&b->step_graph, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    b->step_key = keybuf;
  }
  CK(cudaGraphLaunch(b->step_graph, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  memcpy(u_out, down, b->HM() * 4);
  if (diag3) memcpy(diag3, down + (b->off_diag() - b->off_uout()), 3 * 4);
  return MPPI_OK;
}

int mppi_backend_batch_prepare(mppi_backend* b, uint32_t N, uint32_t T, const float* x0,
                               const float* u_nom, const mppi_batch_agents* agents,
                               uint32_t ws, uint32_t wc, uint32_t wk, uint32_t wt, char* err,
                               size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (N == 0 || T == 0 || !x0) {
    set_err(err, err_len, "num_agents and num_steps must be > 0 and x0 must not be null.");
    return MPPI_ERR_INVALID;
  }
  b->ragged = agents && (agents->sample_counts || agents->horizons);
  if (b->ragged) {
    CK(cudaStreamSynchronize(b->stream));  // the tables below may be in use
    b->agent_K.assign(N, b->K);
    b->agent_H.assign(N, b->H);
    for (uint32_t a = 0; a < N; ++a) {
      if (agents->sample_counts) b->agent_K[a] = agents->sample_counts[a];
      if (agents->horizons) b->agent_H[a] = agents->horizons[a];
      if (b->agent_K[a] == 0 || b->agent_K[a] > b->K) {
        set_err(err, err_len, "sample_counts[" + std::to_string(a) + "] (" +
                                  std::to_string(b->agent_K[a]) +
                                  ") must be in [1, DriverConfig::sample_count = " +
                                  std::to_string(b->K) + "].");
        b->ragged = false;
        return MPPI_ERR_INVALID;
      }
      if (b->agent_H[a] == 0 || b->agent_H[a] > b->H) {
        set_err(err, err_len, "horizons[" + std::to_string(a) + "] (" +
                                  std::to_string(b->agent_H[a]) +
                                  ") must be in [1, DriverConfig::horizon = " +
                                  std::to_string(b->H) + "].");
        b->ragged = false;
        return MPPI_ERR_INVALID;
      }
    }
    // work items, longest horizon first (then more samples first), so the
    // longest items start earliest: list scheduling by decreasing work
    b->agent_blk0.assign(N, 0);
    uint32_t rec = 0;
    std::vector<uint32_t> order(N);
    for (uint32_t a = 0; a < N; ++a) {
      b->agent_blk0[a] = rec;
      rec += (b->agent_K[a] + 127) / 128;
      order[a] = a;
    }
    b->total_records = rec;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      if (b->agent_H[x] != b->agent_H[y]) return b->agent_H[x] > b->agent_H[y];
      return b->agent_K[x] > b->agent_K[y];
    });
    std::vector<uint32_t> work;
    work.reserve(2 * (size_t)rec);
    for (uint32_t a : order)
      for (uint32_t k = 0; k < (b->agent_K[a] + 127) / 128; ++k) {
        work.push_back(a);
        work.push_back(k);
      }
    b->num_work = rec;
    std::vector<uint32_t> info(3 * (size_t)N);
    std::copy(b->agent_K.begin(), b->agent_K.end(), info.begin());
    std::copy(b->agent_H.begin(), b->agent_H.end(), info.begin() + N);
    std::copy(b->agent_blk0.begin(), b->agent_blk0.end(), info.begin() + 2 * N);
    bool grew = false;
    CK(b->d_agent_info.ensure(info.size() * 4, &grew));
    CK(b->d_work.ensure(work.size() * 4, &grew));
    CK(b->d_queue.ensure(16, &grew));
    if (grew) ++b->generation;
    CK(cudaMemcpy(b->d_agent_info.p, info.data(), info.size() * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b->d_work.p, work.data(), work.size() * 4, cudaMemcpyHostToDevice));
  }
  if (int rc = ensure_shape(b, N, T, ws, wc, wk, wt, err, err_len)) return rc;
  b->run_mp = pick_params(b, true, nullptr, 0);
  b->run_cp = pick_params(b, false, nullptr, 0);
  b->run_mp_stride = b->run_cp_stride = 0;
  b->run_sigma = b->c_sigma();
  b->run_sigma_stride = 0;
  if (agents) {
    bool grew = false;
    if (agents->model_params && b->mp_size > 0) {
      const size_t st = pad16(b->mp_size);
      std::vector<uint8_t> tmp(st * N, 0);
      for (uint32_t a = 0; a < N; ++a)
        memcpy(tmp.data() + st * a,
               static_cast<const uint8_t*>(agents->model_params) + agents->model_params_stride * a,
               b->mp_size);
      CK(b->d_agent_mp.ensure(tmp.size(), &grew));
      CK(cudaMemcpy(b->d_agent_mp.p, tmp.data(), tmp.size(), cudaMemcpyHostToDevice));
      b->run_mp = b->d_agent_mp.as<uint8_t>();
      b->run_mp_stride = st;
    }
    if (agents->cost_params && b->cp_size > 0) {
      const size_t st = pad16(b->cp_size);
      std::vector<uint8_t> tmp(st * N, 0);
      for (uint32_t a = 0; a < N; ++a)
        memcpy(tmp.data() + st * a,
               static_cast<const uint8_t*>(agents->cost_params) + agents->cost_params_stride * a,
               b->cp_size);
      CK(b->d_agent_cp.ensure(tmp.size(), &grew));
      CK(cudaMemcpy(b->d_agent_cp.p, tmp.data(), tmp.size(), cudaMemcpyHostToDevice));
      b->run_cp = b->d_agent_cp.as<uint8_t>();
      b->run_cp_stride = st;
    }
    if (agents->sigma) {
      const size_t sl = b->sig_len();
      std::vector<float> tmp(sl * N);
      for (uint32_t a = 0; a < N; ++a) {
        const float* src = agents->sigma + sl * a;
        if (b->cov_full) {
          std::vector<float> L;
          if (!cholesky(b->m, src, &L)) {
            set_err(err, err_len, "per-agent sigma of agent " + std::to_string(a) +
                                      " is not symmetric positive definite.");
            return MPPI_ERR_INVALID;
          }
          std::copy(L.begin(), L.end(), tmp.begin() + sl * a);
        } else {
          std::copy(src, src + sl, tmp.begin() + sl * a);
        }
      }
      CK(b->d_agent_sigma.ensure(tmp.size() * 4, &grew));
      CK(cudaMemcpy(b->d_agent_sigma.p, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice));
      b->run_sigma = b->d_agent_sigma.as<float>();
      b->run_sigma_stride = (uint32_t)sl;
    }
    if (grew) ++b->generation;
  }
  return upload_state(b, 0, x0, u_nom, nullptr, 0, nullptr, 0, err, err_len);
}

int mppi_backend_batch_run(mppi_backend* b, uint64_t start_step, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (b->N == 0 || b->T == 0) {
    set_err(err, err_len, "mppi_backend_batch_run: no batch prepared.");
    return MPPI_ERR_INVALID;
  }
  uint32_t* up = b->h_up.as<uint32_t>();
  CK(cudaStreamSynchronize(b->stream));  // the pinned word may still feed a copy
  up[0] = (uint32_t)start_step;
  CK(cudaMemcpyAsync(b->io(), up, 4, cudaMemcpyHostToDevice, b->stream));
  CK(cudaEventRecord(b->ev0, b->stream));
  if (int rc = enqueue_closed_loop(b, err, err_len)) return rc;
  CK(cudaEventRecord(b->ev1, b->stream));
  b->run_timed = true;
  return MPPI_OK;
}

int mppi_backend_last_run_ms(mppi_backend* b, float* ms, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (!b->run_timed || !ms) {
    set_err(err, err_len, "no closed-loop run has been issued.");
    return MPPI_ERR_INVALID;
  }
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  return MPPI_OK;
}

int mppi_backend_batch_fetch(mppi_backend* b, float* states, float* controls, float* costs,
                             float* terminal, float* x_out, float* u_nom_out, char* err,
                             size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  const size_t N = b->N, T = b->T;
  if (states && b->want_s)
    CK(cudaMemcpyAsync(states, b->d_hs.p, T * N * b->n * 4, cudaMemcpyDeviceToHost, b->stream));
  if (controls && b->want_c)
    CK(cudaMemcpyAsync(controls, b->d_hc.p, T * N * b->m * 4, cudaMemcpyDeviceToHost, b->stream));
  if (costs && b->want_k)
    CK(cudaMemcpyAsync(costs, b->d_hk.p, T * N * 4, cudaMemcpyDeviceToHost, b->stream));
  if (terminal && b->want_t)
    CK(cudaMemcpyAsync(terminal, b->d_term.p, N * b->n * 4, cudaMemcpyDeviceToHost, b->stream));
  if (x_out)
    CK(cudaMemcpyAsync(x_out, b->io() + b->off_x(), N * b->n * 4, cudaMemcpyDeviceToHost,
                       b->stream));
  if (u_nom_out)
    CK(cudaMemcpyAsync(u_nom_out, b->io() + b->off_unom(), N * b->HM() * 4,
                       cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_dispatch_simulation(mppi_backend* b, uint32_t T, uint64_t start_step,
                                     const float* x0, const float* u_nom, const void* mp,
                                     size_t mp_bytes, const void* cp, size_t cp_bytes,
                                     float* states, float* controls, float* costs, char* err,
                                     size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (!u_nom) {
    set_err(err, err_len, "u_nominal must not be null.");
    return MPPI_ERR_INVALID;
  }
  if (int rc = check_override_sizes(b, mp_bytes, mp, cp_bytes, cp, err, err_len)) return rc;
  if (int rc = mppi_backend_batch_prepare(b, 1, T, x0, u_nom, nullptr, states != nullptr,
                                          controls != nullptr, costs != nullptr, false, err,
                                          err_len))
    return rc;
  if ((mp && mp_bytes) || (cp && cp_bytes)) {
    b->run_mp = pick_params(b, true, mp, mp_bytes);
    b->run_cp = pick_params(b, false, cp, cp_bytes);
    if (int rc = upload_state(b, 0, x0, u_nom, mp, mp_bytes, cp, cp_bytes, err, err_len))
      return rc;
  }
  if (int rc = mppi_backend_batch_run(b, start_step, err, err_len)) return rc;
  return mppi_backend_batch_fetch(b, states, controls, costs, nullptr, nullptr, nullptr, err,
                                  err_len);
}

int mppi_backend_dispatch_batch_simulation(mppi_backend* b, uint32_t N, uint32_t T,
                                           uint64_t start_step, const float* x0,
                                           const float* u_nom, const mppi_batch_agents* agents,
                                           float* states, float* controls, float* costs,
                                           float* terminal, char* err, size_t err_len) {
  if (int rc = mppi_backend_batch_prepare(b, N, T, x0, u_nom, agents, states != nullptr,
                                          controls != nullptr, costs != nullptr,
                                          terminal != nullptr, err, err_len))
    return rc;
  if (int rc = mppi_backend_batch_run(b, start_step, err, err_len)) return rc;
  return mppi_backend_batch_fetch(b, states, controls, costs, terminal, nullptr, nullptr, err,
                                  err_len);
}

int mppi_backend_reset(mppi_backend* b, char* err, size_t err_len) {
  if (!b) return MPPI_ERR_INVALID;
  if (!b->initialized) return MPPI_OK;
  if (int rc = check_init(b, err, err_len)) return rc;
  CK(cudaStreamSynchronize(b->stream));
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graph_key.clear();
  b->d_io.release();
  b->d_costs.release();
  b->d_partials.release();
  b->d_hs.release();
  b->d_hc.release();
  b->d_hk.release();
  b->d_term.release();
  b->d_agent_sigma.release();
  b->d_agent_mp.release();
  b->d_agent_cp.release();
  b->N = b->T = 0;
  ++b->generation;
  return MPPI_OK;
}

int mppi_backend_last_costs(mppi_backend* b, uint32_t a0, uint32_t n, float* out, char* err,
                            size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (int rc = check_step_costs(b, a0, n, out, err, err_len)) return rc;
  CK(cudaMemcpyAsync(out, b->d_costs.as<float>() + (size_t)a0 * b->K, (size_t)n * b->K * 4,
                     cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_last_cost_pairs(mppi_backend* b, uint32_t a0, uint32_t n, double* out,
                                 char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (int rc = check_step_costs(b, a0, n, reinterpret_cast<const float*>(out), err, err_len))
    return rc;
  const size_t cnt = (size_t)n * b->K;
  std::vector<float> hi(cnt), lo(cnt);
  const float* base = b->d_costs.as<float>() + (size_t)a0 * b->K;
  CK(cudaMemcpyAsync(hi.data(), base, cnt * 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaMemcpyAsync(lo.data(), base + (size_t)b->N * b->K, cnt * 4, cudaMemcpyDeviceToHost,
                     b->stream));
  CK(cudaStreamSynchronize(b->stream));
  for (size_t i = 0; i < cnt; ++i) out[i] = (double)hi[i] + (double)lo[i];
  return MPPI_OK;
}

int mppi_backend_last_weights(mppi_backend* b, uint32_t a0, uint32_t n, float* out, char* err,
                              size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (int rc = check_step_costs(b, a0, n, out, err, err_len)) return rc;
  DevBuf w;
  CK(w.ensure((size_t)b->N * b->K * 4));
  MppiWeightsArgs a{};
  a.num_agents = b->N;
  a.K = b->K;
  a.lambda = b->lambda;
  a.costs = b->d_costs.as<float>();
  a.costs_lo = a.costs + (size_t)b->N * b->K;
  a.stats = b->io() + b->off_stats();
  a.weights = w.as<float>();
  void* args[] = {&a};
  CK(cudaLaunchKernel((const void*)b->mod->weights, dim3((b->K + 255) / 256, b->N), dim3(256),
                      args, 0, b->stream));
  CK(cudaMemcpyAsync(out, w.as<float>() + (size_t)a0 * b->K, (size_t)n * b->K * 4,
                     cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_sample_noise(mppi_backend* b, uint64_t step, uint32_t agent, uint32_t k0,
                              uint32_t count, const float* sigma, float* normals, float* eps,
                              char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (count == 0) return MPPI_OK;
  const size_t per = (size_t)count * b->HM();
  DevBuf dn, de, ds;
  CK(dn.ensure(per * 4));
  CK(de.ensure(per * 4));
  const float* sig = b->c_sigma();
  if (sigma) {
    std::vector<float> s;
    if (b->cov_full) {
      if (!cholesky(b->m, sigma, &s)) {
        set_err(err, err_len, "sigma is not symmetric positive definite.");
        return MPPI_ERR_INVALID;
      }
    } else {
      s.assign(sigma, sigma + b->m);
    }
    CK(ds.ensure(s.size() * 4));
    CK(cudaMemcpy(ds.p, s.data(), s.size() * 4, cudaMemcpyHostToDevice));
    sig = ds.as<float>();
  }
  MppiNoiseArgs a{};
  a.k0 = k0;
  a.count = count;
  a.H = b->H;
  a.key = b->seed + agent;
  a.step = (uint32_t)step;
  a.sigma = sig;
  a.normals = dn.as<float>();
  a.eps = de.as<float>();
  void* args[] = {&a};
  CK(cudaLaunchKernel((const void*)b->mod->noise, dim3((count + 127) / 128), dim3(128), args, 0,
                      b->stream));
  if (normals) CK(cudaMemcpyAsync(normals, dn.p, per * 4, cudaMemcpyDeviceToHost, b->stream));
  if (eps) CK(cudaMemcpyAsync(eps, de.p, per * 4, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_time_passes(mppi_backend* b, uint32_t iters, float* rollout_ms,
                             float* combine_ms, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (b->N == 0 || iters == 0) {
    set_err(err, err_len, "no batch prepared / iters == 0.");
    return MPPI_ERR_INVALID;
  }
  float ms = 0.0f;
  CK(cudaEventRecord(b->ev0, b->stream));
  for (uint32_t i = 0; i < iters; ++i) CK(launch_rollout_kernel(b, 0));
  CK(cudaEventRecord(b->ev1, b->stream));
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  if (rollout_ms) *rollout_ms = ms / iters;
  CK(cudaEventRecord(b->ev0, b->stream));
  for (uint32_t i = 0; i < iters; ++i) CK(launch_combine(b, 0, false));
  CK(cudaEventRecord(b->ev1, b->stream));
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  if (combine_ms) *combine_ms = ms / iters;
  return MPPI_OK;
}

int mppi_backend_time_proposal(mppi_backend* b, uint32_t iters, float* features_ms,
                               float* network_ms, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (b->N == 0 || iters == 0 || !b->proposal || !b->spec.proposal) {
    set_err(err, err_len, "no proposal attached / no batch prepared / iters == 0.");
    return MPPI_ERR_INVALID;
  }
  float ms = 0.0f;
  if (net_per_agent(b)) {
    // features kernel alone, then the rows kernel on those features (the
    // per-agent network alone)
    CK(cudaEventRecord(b->ev0, b->stream));
    for (uint32_t i = 0; i < iters; ++i) CK(launch_features(b));
    CK(cudaEventRecord(b->ev1, b->stream));
    CK(cudaEventSynchronize(b->ev1));
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (features_ms) *features_ms = ms / iters;
    CK(cudaEventRecord(b->ev0, b->stream));
    for (uint32_t i = 0; i < iters; ++i) CK(launch_proposal_rows(b, true));
    CK(cudaEventRecord(b->ev1, b->stream));
    CK(cudaEventSynchronize(b->ev1));
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    if (network_ms) *network_ms = ms / iters;
    return MPPI_OK;
  }
  CK(cudaEventRecord(b->ev0, b->stream));
  for (uint32_t i = 0; i < iters; ++i) CK(launch_proposal(b));
  CK(cudaEventRecord(b->ev1, b->stream));
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  const float both = ms / iters;
  CK(cudaEventRecord(b->ev0, b->stream));
  for (uint32_t i = 0; i < iters; ++i)
    CK(mppi_b200::proposal_enqueue_forward(b->proposal, b->stream, b->d_feat.as<float>(),
                                           kFeatureStride, b->N, b->d_prop.as<float>()));
  CK(cudaEventRecord(b->ev1, b->stream));
  CK(cudaEventSynchronize(b->ev1));
  CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
  if (network_ms) *network_ms = ms / iters;
  if (features_ms) *features_ms = both - ms / iters;
  return MPPI_OK;
}

int mppi_compile_check(const mppi_backend_plugin* plugin, const mppi_backend_config* cfg,
                       char* log, size_t log_len, char* err, size_t err_len) {
  return mppi_compile_check_proposal(plugin, cfg, 0, nullptr, log, log_len, err, err_len);
}

int mppi_compile_check_proposal(const mppi_backend_plugin* plugin, const mppi_backend_config* cfg,
                                uint32_t proposal, const char* features, char* log,
                                size_t log_len, char* err, size_t err_len) {
  if (!plugin || !cfg) {
    set_err(err, err_len, "null argument.");
    return MPPI_ERR_INVALID;
  }
  mppi_b200::ModuleSpec spec;
  spec.plugin_path = plugin->source_path ? plugin->source_path : "";
  spec.dynamics = plugin->dynamics ? plugin->dynamics : "";
  spec.stage_cost = plugin->stage_cost ? plugin->stage_cost : "";
  spec.terminal_cost = plugin->terminal_cost ? plugin->terminal_cost : "";
  spec.state_dim = cfg->state_dim;
  spec.control_dim = cfg->control_dim;
  spec.cov_full = cfg->covariance_form == 1;
  spec.control_cost = cfg->control_cost != 0;
  spec.noise_half = cfg->numeric_mode != 0;
  spec.model_params_bytes = plugin->model_params_size;
  spec.cost_params_bytes = plugin->cost_params_size;
  spec.model_params_alignment = plugin->model_params_alignment ? plugin->model_params_alignment : 1;
  spec.cost_params_alignment = plugin->cost_params_alignment ? plugin->cost_params_alignment : 1;
  spec.schema_hash = plugin->schema_hash ? plugin->schema_hash : "";
  spec.proposal = proposal != 0;
  spec.features = features ? features : "";
  if (!spec.features.empty() && !valid_identifier(features)) {
    set_err(err, err_len, std::string("Callable '") + features + "' is not a valid identifier.");
    return MPPI_ERR_CALLABLE;
  }
  if (!valid_identifier(spec.dynamics.c_str())) {
    set_err(err, err_len, "Required callable '" + spec.dynamics + "' is not a valid identifier.");
    return MPPI_ERR_CALLABLE;
  }
  std::string lg, e;
  const int rc = mppi_b200::compile_check(spec, &lg, &e);
  set_err(log, log_len, lg);
  if (rc != MPPI_OK) set_err(err, err_len, e);
  return rc;
}

int mppi_backend_tuning_info(mppi_backend* b, uint32_t* grid, uint32_t* num_work,
                             uint32_t* stage_rows, float* rollout_ms) {
  if (!b || !b->initialized) return MPPI_ERR_NOT_INIT;
  if (!b->ragged || b->tuned_key.empty()) return MPPI_ERR_INVALID;
  if (grid) *grid = b->grid;
  if (num_work) *num_work = b->num_work;
  if (stage_rows) *stage_rows = b->geom.stage_rows;
  if (rollout_ms) *rollout_ms = b->tuned_ms;
  return MPPI_OK;
}

int mppi_backend_launch_info(mppi_backend* b, uint32_t* block, uint32_t* nblk,
                             uint32_t* stage_rows, uint32_t* smem_bytes,
                             uint32_t* kernels_per_step) {
  if (!b || !b->initialized) return MPPI_ERR_NOT_INIT;
  if (block) *block = b->geom.block;
  if (nblk) *nblk = b->geom.nblk;
  if (stage_rows) *stage_rows = b->geom.stage_rows;
  if (smem_bytes) *smem_bytes = (uint32_t)b->geom.smem;
  if (kernels_per_step)
    *kernels_per_step = (fused_combine(b) ? 1u : 2u) +
                        (b->proposal && b->spec.proposal && !net_per_agent(b) ? 1u : 0u);
  return MPPI_OK;
}

int mppi_backend_step_form(mppi_backend* b, uint32_t* form) {
  if (!b || !b->initialized) return MPPI_ERR_NOT_INIT;
  if (form) *form = b->form | (b->geom.coop ? 4u : 0u);
  return MPPI_OK;
}

}  // extern "C"

// ---- learned proposal (include/mppi_b200/mppi_backend.h, "proposal") ------

namespace {

// Recompiles the kernel module after a change of b->spec; drops the graph
// and the tuned geometry, which depend on the module.
int reload_module(mppi_backend* b, char* err, size_t err_len) {
  CK(cudaStreamSynchronize(b->stream));
  std::string merr;
  std::shared_ptr<const KernelModule> mod;
  const int rc = mppi_b200::load_module(b->spec, &mod, &merr);
  if (rc != MPPI_OK) {
    set_err(err, err_len, merr);
    return rc;
  }
  b->mod = mod;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->graph_key.clear();
  b->tuned_key.clear();
  ++b->generation;
  return MPPI_OK;
}

}  // namespace

extern "C" {

int mppi_backend_set_features(mppi_backend* b, const char* callable, uint32_t feature_dim,
                              char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  const bool none = callable == nullptr || *callable == '\0';
  if (!none && !valid_identifier(callable)) {
    set_err(err, err_len, std::string("Callable '") + callable + "' is not a valid identifier.");
    return MPPI_ERR_CALLABLE;
  }
  if (!none && (feature_dim == 0 || feature_dim > kFeatureStride)) {
    set_err(err, err_len, "feature_dim must be in [1, 32].");
    return MPPI_ERR_INVALID;
  }
  if (none && b->proposal) {
    set_err(err, err_len, "detach the proposal before removing its feature callable.");
    return MPPI_ERR_INVALID;
  }
  const std::string old = b->spec.features;
  b->spec.features = none ? "" : callable;
  if (int rc = reload_module(b, err, err_len)) {
    b->spec.features = old;
    return rc;
  }
  b->feature_dim = none ? 0 : feature_dim;
  return MPPI_OK;
}

int mppi_backend_features(mppi_backend* b, const float* states, uint32_t rows,
                          uint32_t agents_mod, float* out, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (!b->mod->features || b->feature_dim == 0) {
    set_err(err, err_len, "no feature callable set (mppi_backend_set_features).");
    return MPPI_ERR_INVALID;
  }
  if (rows == 0) return MPPI_OK;
  if (!states || !out || agents_mod == 0) {
    set_err(err, err_len, "states and out must not be null and agents_mod must be > 0.");
    return MPPI_ERR_INVALID;
  }
  const uint8_t* mp;
  const uint8_t* cp;
  uint64_t mps = 0, cps = 0;
  if (b->N > 0 && agents_mod == b->N) {  // the prepared batch's per-agent blobs
    mp = b->run_mp;
    cp = b->run_cp;
    mps = b->run_mp_stride;
    cps = b->run_cp_stride;
  } else if (agents_mod == 1) {  // the bound blobs
    mp = pick_params(b, true, nullptr, 0);
    cp = pick_params(b, false, nullptr, 0);
  } else {
    set_err(err, err_len, "agents_mod must be 1 or the prepared batch's num_agents.");
    return MPPI_ERR_INVALID;
  }
  CK(cudaStreamSynchronize(b->stream));
  DevBuf dx, dout;
  CK(dx.ensure((size_t)rows * b->n * 4));
  CK(dout.ensure((size_t)rows * b->feature_dim * 4));
  CK(cudaMemcpyAsync(dx.p, states, (size_t)rows * b->n * 4, cudaMemcpyHostToDevice, b->stream));
  MppiFeaturesArgs f{};
  f.rows = rows;
  f.agents_mod = agents_mod;
  f.x_stride = b->n;
  f.out_stride = b->feature_dim;
  f.x = dx.as<float>();
  f.model_params = mp;
  f.cost_params = cp;
  f.model_stride = mps;
  f.cost_stride = cps;
  f.out = dout.as<float>();
  void* fa[] = {&f};
  CK(cudaLaunchKernel((const void*)b->mod->features, dim3((rows + 127) / 128), dim3(128), fa, 0,
                      b->stream));
  CK(cudaMemcpyAsync(out, dout.p, (size_t)rows * b->feature_dim * 4, cudaMemcpyDeviceToHost,
                     b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_set_proposal(mppi_backend* b, mppi_proposal* p, uint32_t proposal_samples,
                              char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (p) {
    const mppi_b200::ProposalShape ps = mppi_b200::proposal_shape(p);
    if (b->feature_dim == 0) {
      set_err(err, err_len, "set a feature callable first (mppi_backend_set_features).");
      return MPPI_ERR_INVALID;
    }
    if (ps.control_dim != b->m || ps.input_dim > b->feature_dim) {
      set_err(err, err_len,
              "proposal network shape does not fit: need control_dim == DriverConfig::control_dim "
              "and input_dim <= the feature dimension.");
      return MPPI_ERR_INVALID;
    }
    if (ps.device != b->device) {
      set_err(err, err_len, "proposal network lives on another device.");
      return MPPI_ERR_INVALID;
    }
    if (proposal_samples == 0 || proposal_samples > b->K) {
      set_err(err, err_len, "proposal_samples must be in [1, DriverConfig::sample_count].");
      return MPPI_ERR_INVALID;
    }
  }
  const bool want = p != nullptr;
  if (want != b->spec.proposal) {
    b->spec.proposal = want;
    if (int rc = reload_module(b, err, err_len)) {
      b->spec.proposal = !want;
      return rc;
    }
  }
  CK(cudaStreamSynchronize(b->stream));
  b->proposal = p;
  b->prop_samples = p ? proposal_samples : 0;
  b->N = 0;  // buffers and launch geometry are re-derived by the next prepare
  return MPPI_OK;
}

int mppi_backend_set_record_ustar(mppi_backend* b, uint32_t enable, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  CK(cudaStreamSynchronize(b->stream));
  b->record_ustar = enable != 0;
  b->N = 0;  // takes effect at the next prepare
  return MPPI_OK;
}

int mppi_backend_batch_fetch_ustar(mppi_backend* b, float* out, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (!out || !b->record_ustar || b->N == 0 || b->T == 0) {
    set_err(err, err_len, "no recorded batch: enable mppi_backend_set_record_ustar before prepare.");
    return MPPI_ERR_INVALID;
  }
  CK(cudaMemcpyAsync(out, b->d_hu.p, (size_t)b->T * b->N * b->HM() * 4, cudaMemcpyDeviceToHost,
                     b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return MPPI_OK;
}

int mppi_backend_proposal_stage(mppi_backend* b, float* features_out, float* outputs_out,
                                uint32_t* per_agent, char* err, size_t err_len) {
  if (int rc = check_init(b, err, err_len)) return rc;
  if (b->N == 0 || !b->proposal || !b->spec.proposal) {
    set_err(err, err_len, "no proposal attached / no batch prepared.");
    return MPPI_ERR_INVALID;
  }
  CK(launch_proposal(b));
  if (features_out)
    CK(cudaMemcpyAsync(features_out, b->d_feat.p, (size_t)b->N * kFeatureStride * 4,
                       cudaMemcpyDeviceToHost, b->stream));
  if (outputs_out)
    CK(cudaMemcpyAsync(outputs_out, b->d_prop.p,
                       (size_t)b->N * mppi_b200::proposal_shape(b->proposal).out_stride * 4,
                       cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  if (per_agent) *per_agent = net_per_agent(b) ? 1u : 0u;
  return MPPI_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Single-agent step on caller memory + a caller scratch area (used by the
// allocation-free entry point in csrc/noalloc.cu).  Scratch layout (floats):
//   [0, 16)              zero block: the step_base word reads 0, the step index
//                        travels in step_local
//   [16, .. + nblk * ps) per-CTA partial records
//   [.., + 8)            combine statistics
// The geometry is the one a single-agent dispatch_rollout uses (one agent,
// whatever batch the backend prepared last), so both calls compute the same
// bits.  Per-sample costs are not kept (no inspection on this path).
// ---------------------------------------------------------------------------
#include "step_scratch.hpp"

namespace mppi_b200 {

size_t step_scratch_floats(const mppi_backend* b) {
  const LaunchGeom g = choose_geometry(b, 1);
  return 16 + (size_t)g.nblk * g.pstride + MPPI_STATS_STRIDE;
}

int backend_device(const mppi_backend* b) { return b->device; }
cudaStream_t backend_stream(const mppi_backend* b) { return b->stream; }
bool backend_initialized(const mppi_backend* b) { return b != nullptr && b->initialized; }
bool backend_has_proposal(const mppi_backend* b) { return b->proposal != nullptr; }

int launch_step_with_scratch(mppi_backend* b, uint64_t step_index, const float* x0,
                             const float* u_nominal, const void* model_params,
                             const void* cost_params, float* u_out, float* diag3,
                             float* scratch, size_t scratch_floats, cudaStream_t stream,
                             std::string* error) {
  char ebuf[512] = {0};
  char* err = ebuf;
  const size_t err_len = sizeof(ebuf);
  auto fail = [&](int rc) {
    *error = ebuf;
    return rc;
  };
  const LaunchGeom g = choose_geometry(b, 1);
  const size_t need = step_scratch_floats(b);
  if (scratch_floats < need) {
    *error = "scratch too small";
    return MPPI_ERR_INVALID;
  }
  float* zero = scratch;
  float* partials = scratch + 16;
  float* stats = partials + (size_t)g.nblk * g.pstride;
  const void* rk = g.coop ? (const void*)b->mod->rollout_coop[g.coop_v]
                          : (const void*)b->mod->rollout[g.variant];
  const uint32_t threads = g.coop ? g.block * g.coop : g.block;
  if (g.smem > 48 * 1024) {
    // raise the kernel's dynamic shared memory limit if it is below this
    // launch's need; never lower it (a prepared batch may need more)
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, rk);
    if (e == cudaSuccess && (size_t)fa.maxDynamicSharedSizeBytes < g.smem)
      e = cudaFuncSetAttribute(rk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g.smem);
    if (e != cudaSuccess) {
      set_err(err, err_len, std::string("rollout shared memory limit: ") + cudaGetErrorString(e));
      return fail(MPPI_ERR_CUDA);
    }
  }
  cudaError_t e = cudaMemsetAsync(zero, 0, 16 * sizeof(float), stream);
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    return fail(MPPI_ERR_CUDA);
  }
  MppiRolloutArgs a{};
  a.num_agents = 1;
  a.K = b->K;
  a.H = b->H;
  a.nblk = g.nblk;
  a.stage_rows = g.stage_rows;
  a.seed = b->seed;
  a.step_local = (uint32_t)step_index;
  a.pstride = g.pstride;
  a.lambda = b->lambda;
  a.step_base = reinterpret_cast<const uint32_t*>(zero);
  a.x = x0;
  a.u_nom = u_nominal;
  a.sigma = b->c_sigma();
  a.sigma_inv = b->c_sigma_inv();
  a.u_min = b->c_umin();
  a.u_max = b->c_umax();
  a.model_params = model_params ? static_cast<const uint8_t*>(model_params)
                                : b->d_zero.as<uint8_t>();
  a.cost_params = cost_params ? static_cast<const uint8_t*>(cost_params)
                              : b->d_zero.as<uint8_t>();
  a.partials = partials;
  void* ra[] = {&a};
  e = cudaLaunchKernel(rk, dim3(g.nblk, 1), dim3(threads), ra, g.smem, stream);
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("rollout launch: ") + cudaGetErrorString(e));
    return fail(MPPI_ERR_CUDA);
  }
  MppiCombineArgs c{};
  c.num_agents = 1;
  c.K = b->K;
  c.H = b->H;
  c.nblk = g.nblk;
  c.pstride = g.pstride;
  c.step_local = (uint32_t)step_index;
  c.lambda = b->lambda;
  c.propagate = 0;
  c.step_base = reinterpret_cast<const uint32_t*>(zero);
  c.partials = partials;
  c.u_min = b->c_umin();
  c.u_max = b->c_umax();
  c.model_params = a.model_params;
  c.u_nom = const_cast<float*>(u_nominal);  // read only: propagate == 0
  c.u_out = u_out;
  c.diag = diag3;
  c.stats = stats;
  void* ca[] = {&c};
  e = cudaLaunchKernel((const void*)b->mod->combine, dim3(1), dim3(256), ca,
                       (pad4(g.nblk) + pad4(b->HM())) * 4, stream);
  if (e != cudaSuccess) {
    set_err(err, err_len, std::string("combine launch: ") + cudaGetErrorString(e));
    return fail(MPPI_ERR_CUDA);
  }
  return MPPI_OK;
}

}  // namespace mppi_b200
