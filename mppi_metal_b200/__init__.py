"""mppi_metal_b200 — MPPI (Model Predictive Path Integral) control on NVIDIA
B200 (sm_100a), a drop-in for the rollout -> weights -> update path behind the
``mppi_metal::MPPIDriver`` API of MarshallVielmetti/mppi_metal.

The product is the native library ``lib/libmppi_b200.so`` (C++ driver, C ABI,
NVRTC-compiled CUDA kernels).  This package builds it (``build``) and mirrors
its API for Python callers (``driver``, ``backend``); model-plugin sources and
their parameter layouts live in ``plugins/`` and ``models``.
"""
from .driver import (  # noqa: F401
    BatchAgentParams, BatchSimulationResults, ByteView, CallableNames, ControlBounds,
    ControlNoiseConfig, ControlSequenceView, CovarianceForm, DriverConfig, DriverOptions,
    ErrorRef, ModelPluginSpec, MPPIDriver, MutableControlSequenceView, NumericMode,
    ParamLayout, ProblemParams, RngConfig, SimulationResults, StateView, StepDiagnostics,
    StepInputs)

__version__ = "0.1.0"
