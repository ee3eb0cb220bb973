"""numpy wrapper over the backend C ABI (include/mppi_b200/mppi_backend.h).

The layer under ``MPPIDriver``: one compiled module + device state per
instance.  Tests use it for the per-pass parity checks (costs, weights,
noise) and the benchmark for the device-resident closed loop.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib


class BackendError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
        self.msg = msg


def _f32(a) -> Optional[np.ndarray]:
    if a is None:
        return None
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _p(a):
    return None if a is None else a.ctypes.data


def _check(rc: int, eb) -> None:
    if rc != _lib.MPPI_OK:
        raise BackendError(rc, eb.value.decode(errors="replace"))


def _blob(b: Optional[bytes]):
    if not b:
        return None, 0
    buf = ctypes.create_string_buffer(bytes(b), len(b))
    return ctypes.cast(buf, ctypes.c_void_p), len(b), buf


class Backend:
    """One MPPI problem on the GPU: plugin + config + device buffers."""

    def __init__(self, plugin: str, state_dim: int, control_dim: int, horizon: int,
                 sample_count: int, lam: float, sigma, u_min, u_max, sigma_inv=None,
                 cov_full: bool = False, control_cost: bool = False,
                 stage_cost: str = "mppi_stage_cost", terminal_cost: str = "mppi_terminal_cost",
                 dynamics: str = "mppi_dynamics", model_params_size: int = 0,
                 cost_params_size: int = 0, seed: int = 0, numeric_mode: int = 0,
                 model_params_alignment: int = 1, cost_params_alignment: int = 1,
                 schema_hash: str = ""):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        if self.lib.mppi_backend_create(ctypes.byref(h)) != _lib.MPPI_OK:
            raise MemoryError("mppi_backend_create failed")
        self.h = h
        self.n, self.m, self.H, self.K = state_dim, control_dim, horizon, sample_count
        self.lam = lam
        self.seed = seed
        sig = _f32(sigma)
        sinv = _f32(sigma_inv if sigma_inv is not None else np.zeros_like(sig))
        lo, hi = _f32(u_min), _f32(u_max)
        cfg = _lib.BackendConfig(state_dim, control_dim, horizon, sample_count, lam,
                                 1 if cov_full else 0, _p(sig), _p(sinv), _p(lo), _p(hi),
                                 numeric_mode, 1 if control_cost else 0)
        path = plugin if plugin.endswith(".cu") or "/" in plugin else _lib.plugin_path(plugin)
        plug = _lib.BackendPlugin(path.encode(), dynamics.encode(), stage_cost.encode(),
                                  terminal_cost.encode(), model_params_size, cost_params_size,
                                  seed & 0xFFFFFFFFFFFFFFFF, model_params_alignment,
                                  cost_params_alignment, schema_hash.encode())
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_initialize(self.h, ctypes.byref(plug), ctypes.byref(cfg),
                                                eb, len(eb)), eb)
        self.N = 0
        self.T = 0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mppi_backend_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # -- MetalBackend-shaped calls ----------------------------------------------
    def bind_params(self, model_params: Optional[bytes], cost_params: Optional[bytes]) -> None:
        mp = _blob(model_params)
        cp = _blob(cost_params)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_bind_params(self.h, mp[0], mp[1], cp[0], cp[1], eb, len(eb)),
               eb)

    def dispatch_rollout(self, step: int, x0, u_nom, model_override: Optional[bytes] = None,
                         cost_override: Optional[bytes] = None):
        x0, u_nom = _f32(x0), _f32(u_nom)
        mo, co = _blob(model_override), _blob(cost_override)
        u_out = np.zeros(self.H * self.m, np.float32)
        diag = np.zeros(3, np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_dispatch_rollout(self.h, step, _p(x0), _p(u_nom), mo[0],
                                                      mo[1], co[0], co[1], _p(u_out), _p(diag),
                                                      eb, len(eb)), eb)
        self.N, self.T = 1, 0
        return u_out, diag

    def dispatch_rollout_noalloc(self, step: int, d_x0: int, d_u_nom: int, d_model_params,
                                 d_cost_params, d_u_out: int, d_diag: int) -> None:
        """Allocation-free step on caller-owned DEVICE buffers (raw addresses)."""
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_dispatch_rollout_noalloc(
            self.h, step, d_x0, d_u_nom, d_model_params, d_cost_params, d_u_out, d_diag, eb,
            len(eb)), eb)

    def simulate(self, T: int, start_step: int, x0, u_nom):
        x0, u_nom = _f32(x0), _f32(u_nom)
        st = np.zeros((T, self.n), np.float32)
        ct = np.zeros((T, self.m), np.float32)
        co = np.zeros(T, np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_dispatch_simulation(self.h, T, start_step, _p(x0), _p(u_nom),
                                                         None, 0, None, 0, _p(st), _p(ct), _p(co),
                                                         eb, len(eb)), eb)
        self.N, self.T = 1, T
        return dict(states=st, controls=ct, costs=co)

    def _agents(self, cost_params=None, cost_stride=0, model_params=None, model_stride=0,
                sigma=None, sample_counts=None, horizons=None):
        if cost_params is None and model_params is None and sigma is None \
                and sample_counts is None and horizons is None:
            return None, []
        mp = _blob(model_params)
        cp = _blob(cost_params)
        sg = _f32(sigma)
        ks = None if sample_counts is None else np.ascontiguousarray(sample_counts, np.uint32)
        hs = None if horizons is None else np.ascontiguousarray(horizons, np.uint32)
        ag = _lib.BatchAgents(mp[0], model_stride, cp[0], cost_stride, _p(sg), _p(ks), _p(hs))
        return ag, [mp, cp, sg, ks, hs]

    def prepare(self, N: int, T: int, x0_packed, u_nom_packed=None, cost_params=None,
                cost_stride: int = 0, model_params=None, model_stride: int = 0, sigma=None,
                want_states=True, want_controls=True, want_costs=True, want_terminal=True,
                sample_counts=None, horizons=None):
        x0 = _f32(x0_packed)
        un = _f32(u_nom_packed)
        ag, keep = self._agents(cost_params, cost_stride, model_params, model_stride, sigma,
                                sample_counts, horizons)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_batch_prepare(
            self.h, N, T, _p(x0), _p(un), ctypes.byref(ag) if ag is not None else None,
            int(want_states), int(want_controls), int(want_costs), int(want_terminal), eb,
            len(eb)), eb)
        self.N, self.T = N, T
        self._flags = (want_states, want_controls, want_costs, want_terminal)

    def run(self, start_step: int = 0) -> None:
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_batch_run(self.h, start_step, eb, len(eb)), eb)

    def last_run_ms(self) -> float:
        """Device time of the last run() (CUDA events on the backend stream)."""
        ms = ctypes.c_float()
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_last_run_ms(self.h, ctypes.byref(ms), eb, len(eb)), eb)
        return ms.value

    def fetch(self):
        N, T = self.N, self.T
        ws, wc, wk, wt = self._flags
        st = np.zeros((T, N, self.n), np.float32) if ws else None
        ct = np.zeros((T, N, self.m), np.float32) if wc else None
        co = np.zeros((T, N), np.float32) if wk else None
        te = np.zeros((N, self.n), np.float32) if wt else None
        x = np.zeros((N, self.n), np.float32)
        un = np.zeros((N, self.H * self.m), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_batch_fetch(self.h, _p(st), _p(ct), _p(co), _p(te), _p(x),
                                                 _p(un), eb, len(eb)), eb)
        return dict(states=st, controls=ct, costs=co, terminal=te, x=x, u_nom=un)

    def simulate_batch(self, N: int, T: int, start_step: int, x0_packed, u_nom_packed=None,
                       cost_params=None, cost_stride: int = 0, model_params=None,
                       model_stride: int = 0, sigma=None, sample_counts=None, horizons=None):
        x0 = _f32(x0_packed)
        un = _f32(u_nom_packed)
        ag, keep = self._agents(cost_params, cost_stride, model_params, model_stride, sigma,
                                sample_counts, horizons)
        st = np.zeros((T, N, self.n), np.float32)
        ct = np.zeros((T, N, self.m), np.float32)
        co = np.zeros((T, N), np.float32)
        te = np.zeros((N, self.n), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_dispatch_batch_simulation(
            self.h, N, T, start_step, _p(x0), _p(un),
            ctypes.byref(ag) if ag is not None else None, _p(st), _p(ct), _p(co), _p(te), eb,
            len(eb)), eb)
        self.N, self.T = N, T
        return dict(states=st, controls=ct, costs=co, terminal=te)

    # -- learned proposal -------------------------------------------------------
    def set_features(self, callable_name: Optional[str], feature_dim: int = 0) -> None:
        """Compile the plugin's proposal-feature callable into the module."""
        eb = _lib.err_buf()
        name = callable_name.encode() if callable_name else None
        _check(self.lib.mppi_backend_set_features(self.h, name, feature_dim, eb, len(eb)), eb)
        self.feature_dim = feature_dim if callable_name else 0

    def features(self, states, agents_mod: int = 1) -> np.ndarray:
        """Features of host state rows [rows][n] (row r: agent r % agents_mod)."""
        x = _f32(states).reshape(-1, self.n)
        out = np.zeros((x.shape[0], self.feature_dim), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_features(self.h, _p(x), x.shape[0], agents_mod, _p(out), eb,
                                              len(eb)), eb)
        return out

    def set_proposal(self, net, proposal_samples: int = 0) -> None:
        """Attach a ProposalNet (None detaches); takes effect at the next prepare."""
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_set_proposal(self.h, None if net is None else net.h,
                                                  proposal_samples, eb, len(eb)), eb)
        self._proposal = net  # keep the network alive while attached

    def set_record_ustar(self, enable: bool) -> None:
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_set_record_ustar(self.h, int(enable), eb, len(eb)), eb)

    def fetch_ustar(self) -> np.ndarray:
        """u* of every step of the last recorded batch: [T][N][H][m]."""
        out = np.zeros((self.T, self.N, self.H, self.m), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_batch_fetch_ustar(self.h, _p(out), eb, len(eb)), eb)
        return out

    def proposal_stage(self):
        """Runs the proposal stage on the prepared batch's current states:
        (features [N][32], network outputs [N][stride], per_agent flag)."""
        feat = np.zeros((self.N, 32), np.float32)
        stride = self._proposal.out_stride
        out = np.zeros((self.N, stride), np.float32)
        flag = ctypes.c_uint32()
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_proposal_stage(self.h, _p(feat), _p(out), ctypes.byref(flag),
                                                    eb, len(eb)), eb)
        return feat, out, bool(flag.value)

    # -- inspection ------------------------------------------------------------
    def last_costs(self, a0: int = 0, n: Optional[int] = None) -> np.ndarray:
        n = self.N - a0 if n is None else n
        out = np.zeros((n, self.K), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_last_costs(self.h, a0, n, _p(out), eb, len(eb)), eb)
        return out

    def last_cost_pairs(self, a0: int = 0, n: Optional[int] = None) -> np.ndarray:
        """The last step's per-sample costs exactly (hi + lo pairs as float64)."""
        n = self.N - a0 if n is None else n
        out = np.zeros((n, self.K), np.float64)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_last_cost_pairs(self.h, a0, n, _p(out), eb, len(eb)), eb)
        return out

    def last_weights(self, a0: int = 0, n: Optional[int] = None) -> np.ndarray:
        n = self.N - a0 if n is None else n
        out = np.zeros((n, self.K), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_last_weights(self.h, a0, n, _p(out), eb, len(eb)), eb)
        return out

    def sample_noise(self, step: int, agent: int, k0: int, count: int, sigma=None):
        sg = _f32(sigma)
        nrm = np.zeros((count, self.H, self.m), np.float32)
        eps = np.zeros((count, self.H, self.m), np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_sample_noise(self.h, step, agent, k0, count, _p(sg), _p(nrm),
                                                  _p(eps), eb, len(eb)), eb)
        return nrm, eps

    def time_passes(self, iters: int = 20):
        r = ctypes.c_float()
        c = ctypes.c_float()
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_time_passes(self.h, iters, ctypes.byref(r), ctypes.byref(c),
                                                 eb, len(eb)), eb)
        return r.value, c.value

    def time_proposal(self, iters: int = 20):
        """(features ms, network ms) of one proposal stage on the prepared batch."""
        f, n = ctypes.c_float(), ctypes.c_float()
        eb = _lib.err_buf()
        _check(self.lib.mppi_backend_time_proposal(self.h, iters, ctypes.byref(f),
                                                   ctypes.byref(n), eb, len(eb)), eb)
        return f.value, n.value

    def tuning_info(self) -> dict:
        """Autotuner choice for the prepared uneven batch (after a run)."""
        g, n, r = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        ms = ctypes.c_float()
        rc = self.lib.mppi_backend_tuning_info(self.h, ctypes.byref(g), ctypes.byref(n),
                                               ctypes.byref(r), ctypes.byref(ms))
        if rc != _lib.MPPI_OK:
            return {}
        return {"grid": g.value, "num_work": n.value, "stage_rows": r.value,
                "rollout_ms": ms.value}

    def launch_info(self) -> dict:
        vals = [ctypes.c_uint32() for _ in range(5)]
        self.lib.mppi_backend_launch_info(self.h, *[ctypes.byref(v) for v in vals])
        keys = ["block", "nblk", "stage_rows", "smem_bytes", "kernels_per_step"]
        info = {k: v.value for k, v in zip(keys, vals)}
        f = ctypes.c_uint32()
        self.lib.mppi_backend_step_form(self.h, ctypes.byref(f))
        info["form"] = {"fused_combine": bool(f.value & 1), "warp_specialised": bool(f.value & 2),
                        "cooperative": bool(f.value & 4)}
        return info


def device_philox(c0, c1, key) -> np.ndarray:
    """Philox-2x32-10 words computed by the library's device kernel."""
    lib = _lib.load()
    c0 = np.ascontiguousarray(c0, dtype=np.uint32)
    c1 = np.ascontiguousarray(c1, dtype=np.uint32)
    key = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros((c0.size, 2), np.uint32)
    eb = _lib.err_buf()
    _check(lib.mppi_device_philox(c0.size, _p(c0), _p(c1), _p(key), _p(out), eb, len(eb)), eb)
    return out


def device_sincos(x, quarter: bool = False):
    """(sin, cos) by the library's own device functions: mppi_sincosf of x in
    radians, or (quarter=True) mppi_sincos_quarter, i.e. of pi/2 * x."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    eb = _lib.err_buf()
    _check(lib.mppi_device_sincos(x.size, _p(x), int(bool(quarter)), _p(s), _p(c), eb, len(eb)),
           eb)
    return s, c


def device_log(x):
    """ln x by the library's own device function (mppi_log)."""
    lib = _lib.load()
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros_like(x)
    eb = _lib.err_buf()
    _check(lib.mppi_device_log(x.size, _p(x), _p(out), eb, len(eb)), eb)
    return out


def compile_check(plugin: str, state_dim: int, control_dim: int, cov_full: bool = False,
                  control_cost: bool = False, stage_cost: str = "mppi_stage_cost",
                  terminal_cost: str = "mppi_terminal_cost", dynamics: str = "mppi_dynamics",
                  model_params_size: int = 0, cost_params_size: int = 0,
                  proposal: bool = False, features: Optional[str] = None,
                  numeric_mode: int = 0, model_params_alignment: int = 1,
                  cost_params_alignment: int = 1, schema_hash: str = ""):
    """NVRTC-compile a plugin with the library kernels for sm_100a (no GPU).
    Returns (status, error, log)."""
    lib = _lib.load()
    path = plugin if plugin.endswith(".cu") or "/" in plugin else _lib.plugin_path(plugin)
    plug = _lib.BackendPlugin(path.encode(), dynamics.encode(), stage_cost.encode(),
                              terminal_cost.encode(), model_params_size, cost_params_size, 0,
                              model_params_alignment, cost_params_alignment,
                              schema_hash.encode())
    cfg = _lib.BackendConfig(state_dim, control_dim, 8, 64, 1.0, 1 if cov_full else 0, None, None,
                             None, None, numeric_mode, 1 if control_cost else 0)
    log = ctypes.create_string_buffer(1 << 18)
    eb = _lib.err_buf(1 << 16)
    rc = lib.mppi_compile_check_proposal(ctypes.byref(plug), ctypes.byref(cfg), int(proposal),
                                         features.encode() if features else None, log, len(log),
                                         eb, len(eb))
    return rc, eb.value.decode(errors="replace"), log.value.decode(errors="replace")
