"""The learned sampling proposal (include/mppi_b200/mppi_proposal.h).

``ProposalNet`` wraps the network's C ABI: a 4-layer GELU MLP whose
forward, backward and Adam steps run as the library's sm_100a kernels
(BF16 tcgen05 GEMMs with FP32 accumulation).  Device buffers are torch CUDA
tensors (memory plumbing only; no torch op is on the compute path).
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib, models
from .backend import Backend, BackendError

# The plugins' feature callable and its widths: unicycle 31 (state 5, goal 2,
# 8 obstacles x 3), quadrotor 29 (state 13, 4 obstacles x 4); the network's
# input is padded to 32.
FEATURES_CALLABLE = "mppi_proposal_features"
UNICYCLE_FEATURES = 31
QUADROTOR_FEATURES = 29


def _check(rc: int, eb) -> None:
    if rc != _lib.MPPI_OK:
        raise BackendError(rc, eb.value.decode(errors="replace"))


def _dev_f32(t):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32
            and t.dim() == 2 and t.stride(1) == 1):
        raise TypeError("expected a 2-D float32 CUDA tensor with unit column stride")
    return t


class ProposalNet:
    """Proposal network: features (<= 32) -> predicted u* (H x m) and m log-scales."""

    def __init__(self, input_dim: int, horizon: int, control_dim: int, max_batch: int = 8192,
                 seed: int = 0, log_scale_min: float = -3.0, log_scale_max: float = 1.0):
        self.lib = _lib.load()
        cfg = _lib.ProposalConfig(input_dim, horizon, control_dim, max_batch, seed,
                                  log_scale_min, log_scale_max)
        eb = _lib.err_buf()
        h = self.lib.mppi_proposal_create(ctypes.byref(cfg), eb, len(eb))
        if not h:
            raise BackendError(_lib.MPPI_ERR_INVALID, eb.value.decode(errors="replace"))
        self.h = ctypes.c_void_p(h)
        self.input_dim, self.horizon, self.control_dim = input_dim, horizon, control_dim
        self.max_batch = max_batch
        self.log_scale_min, self.log_scale_max = log_scale_min, log_scale_max
        self.param_count = int(self.lib.mppi_proposal_param_count(self.h))
        self.out_stride = int(self.lib.mppi_proposal_output_stride(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mppi_proposal_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters ----
    def get_params(self) -> np.ndarray:
        out = np.empty(self.param_count, np.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_proposal_get_params(self.h, out.ctypes.data, self.param_count, eb,
                                                 len(eb)), eb)
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32))
        eb = _lib.err_buf()
        _check(self.lib.mppi_proposal_set_params(self.h, p.ctypes.data, p.size, eb, len(eb)), eb)

    # ---- compute (device tensors) ----
    def forward(self, x):
        import torch
        x = _dev_f32(x)
        out = torch.empty((x.shape[0], self.out_stride), device=x.device, dtype=torch.float32)
        eb = _lib.err_buf()
        _check(self.lib.mppi_proposal_forward(self.h, x.data_ptr(), x.stride(0), x.shape[0],
                                              out.data_ptr(), eb, len(eb)), eb)
        return out

    def gradients(self, x, target, index=None):
        """(loss, flat FP32 gradient) over rows `index` (all rows when None)."""
        x, target = _dev_f32(x), _dev_f32(target)
        rows = x.shape[0] if index is None else index.shape[0]
        g = np.empty(self.param_count, np.float32)
        loss = ctypes.c_float()
        eb = _lib.err_buf()
        _check(self.lib.mppi_proposal_gradients(
            self.h, x.data_ptr(), x.stride(0), target.data_ptr(), target.stride(0),
            None if index is None else index.data_ptr(), rows, ctypes.byref(loss),
            g.ctypes.data, eb, len(eb)), eb)
        return float(loss.value), g

    def train_step(self, x, target, index=None, lr: float = 1e-3,
                   want_loss: bool = True) -> Optional[float]:
        x, target = _dev_f32(x), _dev_f32(target)
        rows = x.shape[0] if index is None else index.shape[0]
        loss = ctypes.c_float()
        eb = _lib.err_buf()
        _check(self.lib.mppi_proposal_train_step(
            self.h, x.data_ptr(), x.stride(0), target.data_ptr(), target.stride(0),
            None if index is None else index.data_ptr(), rows, lr,
            ctypes.byref(loss) if want_loss else None, eb, len(eb)), eb)
        return float(loss.value) if want_loss else None

    def last_train_ms(self) -> float:
        return float(self.lib.mppi_proposal_last_train_ms(self.h))

    def fit(self, x, target, epochs: int, batch: int = 8192, lr: float = 1e-3,
            lr_final: Optional[float] = None, seed: int = 0, log_every: int = 0):
        """Mini-batch Adam over (x, target) device tensors; returns the mean
        loss of each epoch.  Learning rate decays geometrically to lr_final."""
        import torch
        rows = x.shape[0]
        batch = min(batch, self.max_batch, rows)
        steps_per_epoch = max(1, rows // batch)
        total = epochs * steps_per_epoch
        gen = torch.Generator(device="cpu").manual_seed(seed)
        decay = 1.0 if lr_final is None else (lr_final / lr) ** (1.0 / max(1, total - 1))
        history, step = [], 0
        for ep in range(epochs):
            perm = torch.randperm(rows, generator=gen).to(torch.int32).to(x.device)
            acc = 0.0
            for s in range(steps_per_epoch):
                idx = perm[s * batch:(s + 1) * batch]
                want = s == steps_per_epoch - 1 or (log_every and s % log_every == 0)
                l = self.train_step(x, target, idx, lr * decay ** step, want_loss=bool(want))
                step += 1
                if l is not None:
                    acc = l
            history.append(acc)
        return history

    def save(self, path: str) -> None:
        np.savez(path, params=self.get_params(), input_dim=self.input_dim,
                 horizon=self.horizon, control_dim=self.control_dim,
                 log_scale_min=self.log_scale_min, log_scale_max=self.log_scale_max)

    @classmethod
    def load(cls, path: str, max_batch: int = 8192) -> "ProposalNet":
        z = np.load(path)
        net = cls(int(z["input_dim"]), int(z["horizon"]), int(z["control_dim"]), max_batch,
                  0, float(z["log_scale_min"]), float(z["log_scale_max"]))
        net.set_params(z["params"])
        return net


# ---------------------------------------------------------------------------
# Data, training and closed-loop evaluation (unicycle among moving obstacles)
# ---------------------------------------------------------------------------
def make_backend(w: models.Workload, sample_count: Optional[int] = None) -> Backend:
    """Backend for a workload; sample_count overrides the workload's K."""
    b = Backend(w.plugin, w.state_dim, w.control_dim, w.horizon,
                sample_count or w.sample_count, w.lam, w.sigma, w.u_min, w.u_max,
                sigma_inv=w.sigma_inv, cov_full=w.cov_full, control_cost=w.control_cost,
                model_params_size=len(w.model_params), cost_params_size=w.cost_stride,
                seed=w.seed, numeric_mode=w.numeric_mode)
    b.bind_params(w.model_params, w.cost_params[0])
    return b


def _prepare(b: Backend, w: models.Workload) -> None:
    b.prepare(w.num_agents, w.num_steps, w.x0, cost_params=w.cost_params_packed,
              cost_stride=w.cost_stride, sigma=w.agent_sigma)


def collect_pairs_for(make_workload, seeds, feature_dim: int, target_steps: Optional[int] = None):
    """(features [R][feature_dim], u* [R][target_steps*m]) from plain-MPPI
    closed loops: one batched run of make_workload(seed) per seed, u* of
    every step recorded on the device, the recorded states featurised by the
    plugin's feature callable.  target_steps keeps the first steps of u*
    (a network may predict fewer steps than the horizon)."""
    feats, targets = [], []
    for seed in seeds:
        w = make_workload(seed)
        N, T, m = w.num_agents, w.num_steps, w.control_dim
        b = make_backend(w)
        b.set_features(FEATURES_CALLABLE, feature_dim)
        b.set_record_ustar(True)
        _prepare(b, w)
        b.run(0)
        r = b.fetch()
        us = b.fetch_ustar()[:, :, :(target_steps or w.horizon)]
        feats.append(b.features(r["states"].reshape(-1, w.state_dim), agents_mod=N))
        targets.append(np.ascontiguousarray(us.reshape(T * N, -1)))
        b.close()
    return np.concatenate(feats), np.concatenate(targets)


def collect_pairs(seeds, agents: int = 1024, steps: int = 300, sample_count: int = 16384,
                  horizon: int = 64):
    """(features [R][31], u* [R][H*m]) from plain-MPPI closed loops of the
    batched unicycle problem, one run of `agents` x `steps` per seed."""
    return collect_pairs_for(
        lambda seed: models.unicycle_batch(seed=seed, N=agents, K=sample_count, H=horizon,
                                           T=steps), seeds, UNICYCLE_FEATURES)


def train(features: np.ndarray, targets: np.ndarray, horizon: int, control_dim: int,
          epochs: int = 30, batch: int = 8192, lr: float = 2e-3, lr_final: float = 5e-5,
          seed: int = 0) -> "tuple[ProposalNet, list]":
    """Trains a proposal network on the GPU with the library's kernels."""
    import torch
    net = ProposalNet(features.shape[1], horizon, control_dim, max_batch=batch, seed=seed)
    x = torch.from_numpy(np.ascontiguousarray(features, np.float32)).cuda()
    y = torch.from_numpy(np.ascontiguousarray(targets, np.float32)).cuda()
    hist = net.fit(x, y, epochs=epochs, batch=batch, lr=lr, lr_final=lr_final, seed=seed)
    return net, hist


def closed_loop(w: models.Workload, net: Optional[ProposalNet] = None,
                proposal_samples: int = 0, sample_count: Optional[int] = None,
                repeats: int = 1) -> dict:
    """Runs the batched closed loop of `w` (optionally with the proposal) and
    returns the executed cost per agent and the device time per run."""
    b = make_backend(w, sample_count)
    if net is not None:
        b.set_features(FEATURES_CALLABLE, net.input_dim)
        b.set_proposal(net, proposal_samples)
    ms = []
    for _ in range(repeats):
        _prepare(b, w)
        b.run(0)
        ms.append(b.last_run_ms())
    r = b.fetch()
    b.set_proposal(None)
    b.close()
    cost = models.executed_cost(w, r["states"], r["controls"], r["terminal"])
    return {"cost": cost, "ms": ms, "states": r["states"], "controls": r["controls"]}


def train_unicycle_proposal(seeds=(100, 101, 102, 103), agents: int = 1024, steps: int = 300,
                            sample_count: int = 16384, horizon: int = 64, epochs: int = 20,
                            batch: int = 8192, seed: int = 0):
    """The configuration's recipe: about 1.2e6 (state features, u*) pairs
    from plain MPPI at K = 16384, H = 64 on batched unicycle runs (1024
    agents x 300 steps per seed), then Adam for `epochs` epochs."""
    X, Y = collect_pairs(seeds, agents=agents, steps=steps, sample_count=sample_count,
                         horizon=horizon)
    net, hist = train(X, Y, horizon, 2, epochs=epochs, batch=batch, seed=seed)
    return net, hist, X.shape[0]


def train_quadrotor_proposal(seeds=(500, 501, 502, 503), agents: int = 256, steps: int = 100,
                             sample_count: int = 65536, horizon: int = 100,
                             net_horizon: int = 60, epochs: int = 30, batch: int = 8192,
                             seed: int = 0):
    """The quadrotor recipe: (features, first net_horizon steps of u*) pairs
    from plain MPPI at K = 65536, H = 100 (4 seeds x 256 agents x 100 steps
    = 102,400 pairs); the network predicts 60 of the 100 steps (H m + m =
    244 outputs), the later steps keep the warm start as their mean."""
    X, Y = collect_pairs_for(
        lambda s: models.quadrotor_batch(seed=s, N=agents, K=sample_count, H=horizon, T=steps),
        seeds, QUADROTOR_FEATURES, target_steps=net_horizon)
    net, hist = train(X, Y, net_horizon, 4, epochs=epochs, batch=batch, seed=seed)
    return net, hist, X.shape[0]


if __name__ == "__main__":
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(description="Train a proposal network on the GPU.")
    ap.add_argument("--out", required=True, help="weights file (.npz)")
    ap.add_argument("--model", choices=["unicycle", "quadrotor"], default="unicycle")
    ap.add_argument("--seeds", default="")
    ap.add_argument("--agents", type=int, default=0)
    ap.add_argument("--epochs", type=int, default=0)
    a = ap.parse_args()
    t0 = time.time()
    kw = {}
    if a.seeds:
        kw["seeds"] = tuple(int(s) for s in a.seeds.split(","))
    if a.agents:
        kw["agents"] = a.agents
    if a.epochs:
        kw["epochs"] = a.epochs
    fn = train_unicycle_proposal if a.model == "unicycle" else train_quadrotor_proposal
    net, hist, pairs = fn(**kw)
    net.save(a.out)
    print(json.dumps({"pairs": pairs, "epochs": len(hist), "final_loss": hist[-1],
                      "seconds": round(time.time() - t0, 1), "out": a.out}))
