"""Python mirror of the ``mppi_metal::MPPIDriver`` API over the C ABI.

Same types, field names, defaults, methods and error convention as the C++
header (include/mppi_metal/mppi_driver.hpp, itself the reference's
include/mppi_metal/mppi_driver.hpp:18-96): every method returns ``bool`` and,
when given an ``ErrorRef``, stores the message in it (the reference's
``std::string* error``).  Arrays are numpy float32 (views are copied, as the
C++ API copies them).
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import _lib


class ErrorRef:
    """Stand-in for ``std::string* error``: receives the failure message."""

    def __init__(self) -> None:
        self.value = ""

    def find(self, needle: str) -> int:
        return self.value.find(needle)

    def __contains__(self, needle: str) -> bool:
        return needle in self.value

    def __str__(self) -> str:
        return self.value


class CovarianceForm(enum.IntEnum):
    kDiagonal = 0
    kFull = 1


class NumericMode(enum.IntEnum):
    kFp32 = 0
    kFp16 = 1
    kMixed = 2


def _f32(a) -> Optional[np.ndarray]:
    if a is None:
        return None
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


@dataclass
class ControlNoiseConfig:
    covariance_form: CovarianceForm = CovarianceForm.kDiagonal
    sigma: Optional[np.ndarray] = None
    sigma_inv: Optional[np.ndarray] = None
    control_dim: int = 0


@dataclass
class ControlBounds:
    u_min: Optional[np.ndarray] = None
    u_max: Optional[np.ndarray] = None
    control_dim: int = 0


@dataclass
class DriverConfig:
    state_dim: int = 0
    control_dim: int = 0
    horizon: int = 0
    sample_count: int = 0
    lambda_: float = 1.0
    noise: ControlNoiseConfig = field(default_factory=ControlNoiseConfig)
    bounds: ControlBounds = field(default_factory=ControlBounds)
    numeric_mode: NumericMode = NumericMode.kFp32


@dataclass
class DriverOptions:
    """Project extensions: the lambda * u^T Sigma^-1 eps control cost, and a
    learned sampling proposal (a mppi_metal_b200.proposal.ProposalNet) that
    draws `proposal_samples` of every step's samples around its prediction."""
    control_cost: bool = False
    proposal: object = None
    proposal_samples: int = 0
    proposal_features: str = "mppi_proposal_features"


@dataclass
class RngConfig:
    seed: int = 0


@dataclass
class CallableNames:
    dynamics: str = "mppi_dynamics"
    stage_cost: str = ""
    terminal_cost: str = ""


@dataclass
class ParamLayout:
    model_params_size: int = 0
    model_params_alignment: int = 1
    cost_params_size: int = 0
    cost_params_alignment: int = 1
    schema_hash: str = ""


@dataclass
class ModelPluginSpec:
    user_metallib_path: str = ""  # CUDA plugin source on this backend
    callables: CallableNames = field(default_factory=CallableNames)
    param_layout: ParamLayout = field(default_factory=ParamLayout)
    rng: RngConfig = field(default_factory=RngConfig)


@dataclass
class ByteView:
    data: Optional[bytes] = None
    bytes: int = 0

    @staticmethod
    def of(blob: Optional[bytes]) -> "ByteView":
        return ByteView(blob, len(blob) if blob else 0)


@dataclass
class ProblemParams:
    model_params: ByteView = field(default_factory=ByteView)
    cost_params: ByteView = field(default_factory=ByteView)


@dataclass
class StateView:
    data: Optional[np.ndarray] = None
    state_dim: int = 0


@dataclass
class ControlSequenceView:
    data: Optional[np.ndarray] = None
    horizon: int = 0
    control_dim: int = 0


@dataclass
class MutableControlSequenceView:
    data: Optional[np.ndarray] = None  # float32, written in place
    horizon: int = 0
    control_dim: int = 0


@dataclass
class StepInputs:
    x0: StateView = field(default_factory=StateView)
    u_nominal_override: ControlSequenceView = field(default_factory=ControlSequenceView)
    model_params_override: ByteView = field(default_factory=ByteView)
    cost_params_override: ByteView = field(default_factory=ByteView)


@dataclass
class StepDiagnostics:
    best_cost: float = 0.0
    mean_cost: float = 0.0
    effective_sample_size: float = 0.0
    converged: bool = False


@dataclass
class SimulationResults:
    states_out: Optional[np.ndarray] = None
    controls_out: Optional[np.ndarray] = None
    costs_out: Optional[np.ndarray] = None
    num_steps: int = 0


@dataclass
class BatchSimulationResults:
    states_out: Optional[np.ndarray] = None
    controls_out: Optional[np.ndarray] = None
    costs_out: Optional[np.ndarray] = None
    terminal_states_out: Optional[np.ndarray] = None
    num_agents: int = 0
    num_steps: int = 0


@dataclass
class BatchAgentParams:
    """Project extension: per-agent blobs (stride bytes apart) and sigma."""
    model_params: Optional[bytes] = None
    model_params_stride: int = 0
    cost_params: Optional[bytes] = None
    cost_params_stride: int = 0
    sigma: Optional[np.ndarray] = None
    sample_counts: Optional[np.ndarray] = None  # uneven batches (uint32 per agent)
    horizons: Optional[np.ndarray] = None


def _out_array(a: Optional[np.ndarray]) -> Optional[np.ndarray]:
    if a is None:
        return None
    if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"] or not a.flags["WRITEABLE"]:
        raise TypeError("output arrays must be writeable C-contiguous float32")
    return a


def _blob(b: Optional[bytes]):
    if not b:
        return None, 0
    buf = ctypes.create_string_buffer(bytes(b), len(b))
    return buf, len(b)


class MPPIDriver:
    """``mppi_metal::MPPIDriver`` through the C ABI (libmppi_b200.so)."""

    def __init__(self, config: DriverConfig, options: Optional[DriverOptions] = None):
        self._lib = _lib.load()
        options = options or DriverOptions()
        self._keep = [_f32(config.noise.sigma), _f32(config.noise.sigma_inv),
                      _f32(config.bounds.u_min), _f32(config.bounds.u_max)]
        c = _lib.DriverConfigC(
            config.state_dim, config.control_dim, config.horizon, config.sample_count,
            config.lambda_, int(config.noise.covariance_form), _ptr(self._keep[0]),
            _ptr(self._keep[1]), config.noise.control_dim, _ptr(self._keep[2]),
            _ptr(self._keep[3]), config.bounds.control_dim, int(config.numeric_mode),
            int(options.control_cost),
            None if options.proposal is None else options.proposal.h,
            int(options.proposal_samples), options.proposal_features.encode())
        self._proposal = options.proposal  # keep the network alive
        self._h = self._lib.mppi_driver_create(ctypes.byref(c))
        if not self._h:
            raise MemoryError("mppi_driver_create failed")
        self.config = config
        self._keep = None  # the driver deep-copied the arrays

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.mppi_driver_destroy(h)
            self._h = None

    @staticmethod
    def _done(rc: int, buf, error: Optional[ErrorRef]) -> bool:
        if not rc and error is not None:
            error.value = buf.value.decode(errors="replace")
        return bool(rc)

    def initialize(self, model: ModelPluginSpec, error: Optional[ErrorRef] = None) -> bool:
        p = _lib.DriverPluginC(
            str(model.user_metallib_path).encode(), model.callables.dynamics.encode(),
            model.callables.stage_cost.encode(), model.callables.terminal_cost.encode(),
            model.param_layout.model_params_size, model.param_layout.model_params_alignment,
            model.param_layout.cost_params_size, model.param_layout.cost_params_alignment,
            model.param_layout.schema_hash.encode(), model.rng.seed & 0xFFFFFFFFFFFFFFFF)
        eb = _lib.err_buf()
        return self._done(self._lib.mppi_driver_initialize(self._h, ctypes.byref(p), eb, len(eb)),
                          eb, error)

    def set_problem_params(self, params: ProblemParams, error: Optional[ErrorRef] = None) -> bool:
        mp, _ = _blob(params.model_params.data)
        cp, _ = _blob(params.cost_params.data)
        eb = _lib.err_buf()
        rc = self._lib.mppi_driver_set_problem_params(
            self._h, ctypes.cast(mp, ctypes.c_void_p) if mp is not None else None,
            params.model_params.bytes, ctypes.cast(cp, ctypes.c_void_p) if cp is not None else None,
            params.cost_params.bytes, eb, len(eb))
        return self._done(rc, eb, error)

    def step(self, inputs: StepInputs, u_next_out: MutableControlSequenceView,
             diagnostics: Optional[StepDiagnostics] = None,
             error: Optional[ErrorRef] = None) -> bool:
        x0 = _f32(inputs.x0.data)
        ov = _f32(inputs.u_nominal_override.data)
        mo, _ = _blob(inputs.model_params_override.data)
        co, _ = _blob(inputs.cost_params_override.data)
        out = _out_array(u_next_out.data)
        diag = np.zeros(4, np.float32) if diagnostics is not None else None
        eb = _lib.err_buf()
        rc = self._lib.mppi_driver_step(
            self._h, _ptr(x0), inputs.x0.state_dim, _ptr(ov),
            inputs.u_nominal_override.horizon, inputs.u_nominal_override.control_dim,
            ctypes.cast(mo, ctypes.c_void_p) if mo is not None else None,
            inputs.model_params_override.bytes,
            ctypes.cast(co, ctypes.c_void_p) if co is not None else None,
            inputs.cost_params_override.bytes, _ptr(out), u_next_out.horizon,
            u_next_out.control_dim, _ptr(diag), eb, len(eb))
        if rc and diagnostics is not None:
            diagnostics.best_cost = float(diag[0])
            diagnostics.mean_cost = float(diag[1])
            diagnostics.effective_sample_size = float(diag[2])
            diagnostics.converged = bool(diag[3])
        return self._done(rc, eb, error)

    def reset(self, u_nominal: Optional[ControlSequenceView] = None,
              error: Optional[ErrorRef] = None) -> bool:
        eb = _lib.err_buf()
        if u_nominal is None:
            return self._done(self._lib.mppi_driver_reset(self._h, eb, len(eb)), eb, error)
        u = _f32(u_nominal.data)
        rc = self._lib.mppi_driver_reset_nominal(self._h, _ptr(u), u_nominal.horizon,
                                                 u_nominal.control_dim, eb, len(eb))
        return self._done(rc, eb, error)

    def simulate(self, num_steps: int, inputs: StepInputs, results: SimulationResults,
                 error: Optional[ErrorRef] = None) -> bool:
        x0 = _f32(inputs.x0.data)
        ov = _f32(inputs.u_nominal_override.data)
        mo, _ = _blob(inputs.model_params_override.data)
        co, _ = _blob(inputs.cost_params_override.data)
        eb = _lib.err_buf()
        rc = self._lib.mppi_driver_simulate(
            self._h, num_steps, _ptr(x0), inputs.x0.state_dim, _ptr(ov),
            inputs.u_nominal_override.horizon, inputs.u_nominal_override.control_dim,
            ctypes.cast(mo, ctypes.c_void_p) if mo is not None else None,
            inputs.model_params_override.bytes,
            ctypes.cast(co, ctypes.c_void_p) if co is not None else None,
            inputs.cost_params_override.bytes, _ptr(_out_array(results.states_out)),
            _ptr(_out_array(results.controls_out)), _ptr(_out_array(results.costs_out)),
            results.num_steps, eb, len(eb))
        return self._done(rc, eb, error)

    def simulate_batch(self, num_agents: int, num_steps: int, x0_packed,
                       results: BatchSimulationResults,
                       agent_params: Optional[BatchAgentParams] = None,
                       error: Optional[ErrorRef] = None) -> bool:
        x0 = _f32(x0_packed)
        eb = _lib.err_buf()
        outs = [_ptr(_out_array(results.states_out)), _ptr(_out_array(results.controls_out)),
                _ptr(_out_array(results.costs_out)),
                _ptr(_out_array(results.terminal_states_out))]
        if agent_params is None:
            rc = self._lib.mppi_driver_simulate_batch(
                self._h, num_agents, num_steps, _ptr(x0), *outs, results.num_agents,
                results.num_steps, eb, len(eb))
        else:
            mp, _ = _blob(agent_params.model_params)
            cp, _ = _blob(agent_params.cost_params)
            sg = _f32(agent_params.sigma)
            ks = None if agent_params.sample_counts is None else \
                np.ascontiguousarray(agent_params.sample_counts, dtype=np.uint32)
            hs = None if agent_params.horizons is None else \
                np.ascontiguousarray(agent_params.horizons, dtype=np.uint32)
            rc = self._lib.mppi_driver_simulate_batch_agents(
                self._h, num_agents, num_steps, _ptr(x0),
                ctypes.cast(mp, ctypes.c_void_p) if mp is not None else None,
                agent_params.model_params_stride,
                ctypes.cast(cp, ctypes.c_void_p) if cp is not None else None,
                agent_params.cost_params_stride, _ptr(sg), _ptr(ks), _ptr(hs), *outs,
                results.num_agents, results.num_steps, eb, len(eb))
        return self._done(rc, eb, error)
