"""numpy front end for the checkers.  TEST INFRASTRUCTURE ONLY.

Two CPU implementations of the reference MPPI hot path:

* ``Oracle`` — the FP64 C restatement in ``oracle/mppi_oracle.c``
  (``oracle/build/libmppi_oracle.so``).
* ``RefKernels`` — the reference's own Metal kernels compiled for the CPU
  (``oracle/_ref/libmppi_ref_<plugin>.so``, see ``oracle/Makefile``), FP32,
  replaying ``src/metal_backend.mm``'s dispatch sequences.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import
this module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "build" / "libmppi_oracle.so"
REF_DIR = HERE / "_ref"

MODEL_IDS = {
    "double_integrator": 0,
    "nonholonomic_vehicle": 1,
    "unicycle_obstacles": 2,
    "bicycle_lane": 3,
    "quadrotor": 4,
    "gust_integrator": 5,
    "wez_environment": 6,
}

# Which oracle/_ref library runs the reference kernels for each model.
REF_PLUGIN_LIBS = {
    "double_integrator": "test_user_dynamics",
    "nonholonomic_vehicle": "nonholonomic_vehicle",
    "unicycle_obstacles": "unicycle_obstacles",
}

_P = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64


def build_oracle(ref_root: str | os.PathLike | None = None) -> None:
    """Compile the FP64 oracle and, when the reference source tree is given
    (``ref_root``, else the MPPI_REF_ROOT environment variable) and holds the
    reference's shaders, the reference CPU libraries, with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    root = ref_root if ref_root is not None else os.environ.get("MPPI_REF_ROOT", "")
    if not root:
        return
    ref_root = Path(root)
    if (ref_root / "shaders" / "mppi_rollout.metal").exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_ROOT={ref_root}"], check=True)
        product = HERE.parent / "mppi_metal_b200" / "lib" / "libmppi_b200.so"
        if product.exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "ref_suite", "ref_examples",
                            f"REF_ROOT={ref_root}"], check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else _P(a.ctypes.data)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


class _OracleProblem(ctypes.Structure):
    _fields_ = [
        ("state_dim", _u32), ("control_dim", _u32), ("horizon", _u32), ("sample_count", _u32),
        ("lambda_", ctypes.c_double),
        ("cov_full", ctypes.c_int32), ("control_cost", ctypes.c_int32), ("model", ctypes.c_int32),
        ("use_stage", ctypes.c_int32), ("use_terminal", ctypes.c_int32),
        ("noise_half", ctypes.c_int32),
        ("sigma", _P), ("sigma_inv", _P), ("u_min", _P), ("u_max", _P),
        ("model_params", _P), ("cost_params", _P),
    ]


class _AgentInputs(ctypes.Structure):
    _fields_ = [("model_params", _P), ("model_stride", _u64), ("cost_params", _P),
                ("cost_stride", _u64), ("sigma", _P)]


@dataclass
class Problem:
    """One MPPI problem, in the driver's terms (DriverConfig + plugin)."""

    model: str
    state_dim: int
    control_dim: int
    horizon: int
    sample_count: int
    lam: float
    sigma: np.ndarray
    u_min: np.ndarray
    u_max: np.ndarray
    sigma_inv: np.ndarray | None = None
    cov_full: bool = False
    control_cost: bool = False
    use_stage: bool = True
    use_terminal: bool = True
    noise_half: bool = False
    model_params: bytes = b""
    cost_params: bytes = b""
    _keep: list = field(default_factory=list, repr=False)


class Oracle:
    """FP64 restatement (oracle/mppi_oracle.c)."""

    def __init__(self, path: Path = ORACLE_LIB):
        if not path.exists():
            build_oracle()
        self.lib = ctypes.CDLL(str(path))

    # -- helpers ----------------------------------------------------------
    def _prob(self, p: Problem) -> _OracleProblem:
        keep = []

        def arr(x):
            if x is None:
                return None
            a = _f64(x)
            keep.append(a)
            return _ptr(a)

        def blob(b):
            if not b:
                return None
            buf = ctypes.create_string_buffer(bytes(b), len(b))
            keep.append(buf)
            return ctypes.cast(buf, _P)

        sigma_inv = p.sigma_inv if p.sigma_inv is not None else np.zeros_like(np.asarray(p.sigma))
        s = _OracleProblem(p.state_dim, p.control_dim, p.horizon, p.sample_count, p.lam,
                           int(p.cov_full), int(p.control_cost), MODEL_IDS[p.model],
                           int(p.use_stage), int(p.use_terminal), int(p.noise_half),
                           arr(p.sigma), arr(sigma_inv), arr(p.u_min), arr(p.u_max),
                           blob(p.model_params), blob(p.cost_params))
        s._keep = keep
        return s

    # -- RNG -----------------------------------------------------------------
    def philox(self, c0, c1, key) -> np.ndarray:
        c0 = np.ascontiguousarray(c0, dtype=np.uint32)
        c1 = np.ascontiguousarray(c1, dtype=np.uint32)
        key = np.ascontiguousarray(key, dtype=np.uint32)
        out = np.zeros((c0.size, 2), dtype=np.uint32)
        self.lib.oracle_philox_many(_u64(c0.size), _ptr(c0), _ptr(c1), _ptr(key), _ptr(out))
        return out

    def box_muller(self, words: np.ndarray) -> np.ndarray:
        words = np.asarray(words, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros((words.shape[0], 2))
        buf = (ctypes.c_double * 2)()
        for i, (a, b) in enumerate(words):
            self.lib.oracle_box_muller(_u32(int(a)), _u32(int(b)), buf)
            out[i] = buf[0], buf[1]
        return out

    def noise(self, p: Problem, step: int, key: int, k: int, sigma=None):
        s = self._prob(p)
        sig = _f64(p.sigma if sigma is None else sigma)
        n = np.zeros((p.horizon, p.control_dim))
        e = np.zeros((p.horizon, p.control_dim))
        self.lib.oracle_sample_noise(ctypes.byref(s), _u32(step), _u32(key), _u32(k), _ptr(sig),
                                     _ptr(n), _ptr(e))
        return n, e

    # -- passes ----------------------------------------------------------------
    def rollout(self, p: Problem, step: int, key: int, x0, u_nom, sigma=None,
                model_params: bytes | None = None, cost_params: bytes | None = None):
        s = self._prob(p)
        x0 = _f64(x0)
        u_nom = _f64(u_nom)
        sig = _f64(p.sigma if sigma is None else sigma)
        mp = ctypes.create_string_buffer(model_params or p.model_params or b"\0", max(1, len(model_params or p.model_params or b"\0")))
        cp = ctypes.create_string_buffer(cost_params or p.cost_params or b"\0", max(1, len(cost_params or p.cost_params or b"\0")))
        costs = np.zeros(p.sample_count)
        self.lib.oracle_rollout(ctypes.byref(s), _u32(step), _u32(key), _ptr(x0), _ptr(u_nom),
                                _ptr(sig), mp, cp, _ptr(costs))
        return costs

    def rollout_eps(self, p: Problem, x0, u_nom, eps_all):
        """Rollout costs on a given noise array [K][H][m]."""
        s = self._prob(p)
        x0, u_nom, eps = _f64(x0), _f64(u_nom), _f64(eps_all)
        mp = ctypes.create_string_buffer(p.model_params or b"\0", max(1, len(p.model_params)))
        cp = ctypes.create_string_buffer(p.cost_params or b"\0", max(1, len(p.cost_params)))
        costs = np.zeros(p.sample_count)
        self.lib.oracle_rollout_eps(ctypes.byref(s), _ptr(x0), _ptr(u_nom), mp, cp, _ptr(eps),
                                    _ptr(costs))
        return costs

    def update_eps(self, p: Problem, weights, u_nom, eps_all):
        s = self._prob(p)
        w, u_nom, eps = _f64(weights), _f64(u_nom), _f64(eps_all)
        out = np.zeros(p.horizon * p.control_dim)
        self.lib.oracle_update_eps(ctypes.byref(s), _ptr(w), _ptr(u_nom), _ptr(eps), _ptr(out))
        return out

    def dynamics(self, p: Problem, x, u, step: int = 0, key: int = 0) -> np.ndarray:
        """One step x <- f(x, u) of the problem's model in double, with the
        propagate's counter (step, 0x80000000) and the given key."""
        s = self._prob(p)
        xo = _f64(x).copy()
        u = _f64(u)
        mp = ctypes.create_string_buffer(p.model_params or b"\0", max(1, len(p.model_params)))
        self.lib.oracle_dynamics(ctypes.byref(s), _ptr(xo), _ptr(u), mp, _u32(step),
                                 _u32(0x80000000), _u32(key))
        return xo

    def weights(self, costs, lam: float):
        costs = _f64(costs)
        w = np.zeros(costs.size)
        diag = np.zeros(3)
        self.lib.oracle_weights(_u32(costs.size), ctypes.c_double(lam), _ptr(costs), _ptr(w),
                                _ptr(diag))
        return w, diag

    def update(self, p: Problem, step: int, key: int, weights, u_nom, sigma=None):
        s = self._prob(p)
        w = _f64(weights)
        u_nom = _f64(u_nom)
        sig = _f64(p.sigma if sigma is None else sigma)
        out = np.zeros(p.horizon * p.control_dim)
        self.lib.oracle_update(ctypes.byref(s), _u32(step), _u32(key), _ptr(w), _ptr(u_nom),
                               _ptr(sig), _ptr(out))
        return out

    def step(self, p: Problem, step: int, key: int, x0, u_nom):
        s = self._prob(p)
        x0 = _f64(x0)
        u_nom = _f64(u_nom)
        u_out = np.zeros(p.horizon * p.control_dim)
        diag = np.zeros(3)
        costs = np.zeros(p.sample_count)
        w = np.zeros(p.sample_count)
        self.lib.oracle_step(ctypes.byref(s), _u32(step), _u32(key), _ptr(x0), _ptr(u_nom),
                             _ptr(u_out), _ptr(diag), _ptr(costs), _ptr(w))
        return dict(u_out=u_out, diag=diag, costs=costs, weights=w)

    def simulate(self, p: Problem, T: int, start_step: int, key: int, x0, u_nom0):
        s = self._prob(p)
        x0 = _f64(x0)
        u_nom0 = _f64(u_nom0)
        st = np.zeros((T, p.state_dim))
        ct = np.zeros((T, p.control_dim))
        co = np.zeros(T)
        xf = np.zeros(p.state_dim)
        uf = np.zeros(p.horizon * p.control_dim)
        self.lib.oracle_simulate(ctypes.byref(s), _u32(T), _u32(start_step), _u32(key), _ptr(x0),
                                 _ptr(u_nom0), _ptr(st), _ptr(ct), _ptr(co), _ptr(xf), _ptr(uf))
        return dict(states=st, controls=ct, costs=co, x_final=xf, u_nom_final=uf)

    def simulate_batch(self, p: Problem, N: int, T: int, start_step: int, seed: int, x0_packed,
                       u_nom0_packed=None, cost_params_packed: bytes | None = None,
                       cost_stride: int = 0, model_params_packed: bytes | None = None,
                       model_stride: int = 0, sigma_packed=None):
        s = self._prob(p)
        x0 = _f64(x0_packed)
        un = None if u_nom0_packed is None else _f64(u_nom0_packed)
        keep = []
        ai = None
        if cost_params_packed or model_params_packed or sigma_packed is not None:
            def blob(b):
                if not b:
                    return None
                buf = ctypes.create_string_buffer(bytes(b), len(b))
                keep.append(buf)
                return ctypes.cast(buf, _P)
            sg = None if sigma_packed is None else _f64(sigma_packed)
            keep.append(sg)
            ai = _AgentInputs(blob(model_params_packed), model_stride, blob(cost_params_packed),
                              cost_stride, _ptr(sg))
        st = np.zeros((T, N, p.state_dim))
        ct = np.zeros((T, N, p.control_dim))
        co = np.zeros((T, N))
        term = np.zeros((N, p.state_dim))
        self.lib.oracle_simulate_batch(ctypes.byref(s), _u32(N), _u32(T), _u32(start_step),
                                       _u32(seed), None if ai is None else ctypes.byref(ai),
                                       _ptr(x0), _ptr(un), _ptr(st), _ptr(ct), _ptr(co),
                                       _ptr(term))
        return dict(states=st, controls=ct, costs=co, terminal=term)


class _RefConfig(ctypes.Structure):
    _fields_ = [("state_dim", _u32), ("control_dim", _u32), ("horizon", _u32),
                ("sample_count", _u32), ("lambda_", ctypes.c_float), ("seed", _u32),
                ("use_stage", ctypes.c_int32), ("use_terminal", ctypes.c_int32),
                ("nthreads", ctypes.c_int32), ("pad", ctypes.c_int32)]


def ref_available(model: str) -> bool:
    name = REF_PLUGIN_LIBS.get(model)
    return name is not None and (REF_DIR / f"libmppi_ref_{name}.so").exists()


class RefKernels:
    """The reference's own kernels on the CPU (FP32), for one model plugin."""

    def __init__(self, model: str):
        name = REF_PLUGIN_LIBS[model]
        path = REF_DIR / f"libmppi_ref_{name}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} (build with `make -C oracle ref`)")
        self.lib = ctypes.CDLL(str(path))
        self.model = model

    def _cfg(self, p: Problem, seed: int, nthreads: int) -> _RefConfig:
        return _RefConfig(p.state_dim, p.control_dim, p.horizon, p.sample_count, p.lam,
                          seed & 0xFFFFFFFF, int(p.use_stage), int(p.use_terminal), nthreads, 0)

    def philox(self, c0, c1, key) -> np.ndarray:
        c0 = np.ascontiguousarray(c0, dtype=np.uint32)
        c1 = np.ascontiguousarray(c1, dtype=np.uint32)
        key = np.ascontiguousarray(key, dtype=np.uint32)
        out = np.zeros((c0.size, 2), dtype=np.uint32)
        self.lib.ref_philox_words(_u64(c0.size), _ptr(c0), _ptr(c1), _ptr(key), _ptr(out))
        return out

    def box_muller(self, words) -> np.ndarray:
        words = np.ascontiguousarray(words, dtype=np.uint32).reshape(-1, 2)
        out = np.zeros(words.shape, dtype=np.float32)
        self.lib.ref_box_muller(_u64(words.shape[0]), _ptr(words), _ptr(out))
        return out

    @staticmethod
    def _blob(b: bytes):
        return ctypes.create_string_buffer(bytes(b), len(b)) if b else None

    def step(self, p: Problem, step: int, seed: int, x0, u_nom, nthreads: int = 1):
        c = self._cfg(p, seed, nthreads)
        x0, u_nom = _f32(x0), _f32(u_nom)
        sig, lo, hi = _f32(p.sigma), _f32(p.u_min), _f32(p.u_max)
        mp, cp = self._blob(p.model_params), self._blob(p.cost_params)
        u_out = np.zeros(p.horizon * p.control_dim, np.float32)
        diag = np.zeros(3, np.float32)
        costs = np.zeros(p.sample_count, np.float32)
        w = np.zeros(p.sample_count, np.float32)
        self.lib.ref_step(ctypes.byref(c), _u32(step), _ptr(x0), _ptr(u_nom), _ptr(sig), _ptr(lo),
                          _ptr(hi), mp, cp, _ptr(u_out), _ptr(diag), _ptr(costs), _ptr(w))
        return dict(u_out=u_out, diag=diag, costs=costs, weights=w)

    def simulate(self, p: Problem, T: int, start_step: int, seed: int, x0, u_nom0,
                 nthreads: int = 1):
        c = self._cfg(p, seed, nthreads)
        x0, u_nom0 = _f32(x0), _f32(u_nom0)
        sig, lo, hi = _f32(p.sigma), _f32(p.u_min), _f32(p.u_max)
        mp, cp = self._blob(p.model_params), self._blob(p.cost_params)
        st = np.zeros((T, p.state_dim), np.float32)
        ct = np.zeros((T, p.control_dim), np.float32)
        co = np.zeros(T, np.float32)
        self.lib.ref_simulate(ctypes.byref(c), _u32(T), _u32(start_step), _ptr(x0), _ptr(u_nom0),
                              _ptr(sig), _ptr(lo), _ptr(hi), mp, cp, _ptr(st), _ptr(ct), _ptr(co))
        return dict(states=st, controls=ct, costs=co)

    def simulate_batch(self, p: Problem, N: int, T: int, start_step: int, seed: int, x0_packed,
                       u_nom0_packed=None, sigma_packed=None, cost_params_packed: bytes = b"",
                       cost_stride: int = 0, model_params_packed: bytes = b"",
                       model_stride: int = 0, nthreads: int = 1):
        c = self._cfg(p, seed, nthreads)
        x0 = _f32(x0_packed)
        un = None if u_nom0_packed is None else _f32(u_nom0_packed)
        if sigma_packed is None:
            sig, sig_stride = _f32(p.sigma), 0
        else:
            sig = _f32(sigma_packed)
            sig_stride = p.control_dim
        lo, hi = _f32(p.u_min), _f32(p.u_max)
        mp = self._blob(model_params_packed or p.model_params)
        cp = self._blob(cost_params_packed or p.cost_params)
        st = np.zeros((T, N, p.state_dim), np.float32)
        ct = np.zeros((T, N, p.control_dim), np.float32)
        co = np.zeros((T, N), np.float32)
        term = np.zeros((N, p.state_dim), np.float32)
        self.lib.ref_simulate_batch(
            ctypes.byref(c), _u32(N), _u32(T), _u32(start_step), _ptr(x0), _ptr(un), _ptr(sig),
            _u64(sig_stride), _ptr(lo), _ptr(hi), mp, _u64(model_stride if model_params_packed else 0),
            cp, _u64(cost_stride if cost_params_packed else 0), _ptr(st), _ptr(ct), _ptr(co),
            _ptr(term))
        return dict(states=st, controls=ct, costs=co, terminal=term)
