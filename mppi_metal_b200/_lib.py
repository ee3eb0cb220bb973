"""Loader and ctypes declarations for libmppi_b200.so (the C ABI in include/).

The product path is the compiled library; there is no Python or CPU fallback:
importing a symbol from a missing library raises immediately.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libmppi_b200.so"
PLUGIN_DIR = PKG / "plugins"
INCLUDE_DIR = PKG.parent / "include"

c_u32 = ctypes.c_uint32
c_u64 = ctypes.c_uint64
c_f32 = ctypes.c_float
c_ptr = ctypes.c_void_p
c_char_p = ctypes.c_char_p
c_size = ctypes.c_size_t

MPPI_OK = 0
MPPI_ERR_INVALID = 1
MPPI_ERR_PLUGIN = 2
MPPI_ERR_CALLABLE = 3
MPPI_ERR_CUDA = 4
MPPI_ERR_NO_DEVICE = 5
MPPI_ERR_NOT_INIT = 6


class BackendConfig(ctypes.Structure):
    """mppi_backend_config (include/mppi_b200/mppi_backend.h)."""
    _fields_ = [
        ("state_dim", c_u32), ("control_dim", c_u32), ("horizon", c_u32),
        ("sample_count", c_u32), ("lambda_", c_f32), ("covariance_form", c_u32),
        ("sigma", c_ptr), ("sigma_inv", c_ptr), ("u_min", c_ptr), ("u_max", c_ptr),
        ("numeric_mode", c_u32), ("control_cost", c_u32),
    ]


class BackendPlugin(ctypes.Structure):
    """mppi_backend_plugin."""
    _fields_ = [
        ("source_path", c_char_p), ("dynamics", c_char_p), ("stage_cost", c_char_p),
        ("terminal_cost", c_char_p), ("model_params_size", c_u64),
        ("cost_params_size", c_u64), ("seed", c_u64),
        ("model_params_alignment", c_u64), ("cost_params_alignment", c_u64),
        ("schema_hash", c_char_p),
    ]


class BatchAgents(ctypes.Structure):
    """mppi_batch_agents."""
    _fields_ = [
        ("model_params", c_ptr), ("model_params_stride", c_u64),
        ("cost_params", c_ptr), ("cost_params_stride", c_u64), ("sigma", c_ptr),
        ("sample_counts", c_ptr), ("horizons", c_ptr),
    ]


class DriverConfigC(ctypes.Structure):
    """mppi_driver_config (include/mppi_b200/mppi_driver_c.h)."""
    _fields_ = [
        ("state_dim", c_u32), ("control_dim", c_u32), ("horizon", c_u32),
        ("sample_count", c_u32), ("lambda_", c_f32), ("covariance_form", c_u32),
        ("sigma", c_ptr), ("sigma_inv", c_ptr), ("noise_control_dim", c_u32),
        ("u_min", c_ptr), ("u_max", c_ptr), ("bounds_control_dim", c_u32),
        ("numeric_mode", c_u32), ("control_cost", c_u32), ("proposal", c_ptr),
        ("proposal_samples", c_u32), ("proposal_features", c_char_p),
    ]


class DriverPluginC(ctypes.Structure):
    """mppi_driver_plugin."""
    _fields_ = [
        ("source_path", c_char_p), ("dynamics", c_char_p), ("stage_cost", c_char_p),
        ("terminal_cost", c_char_p), ("model_params_size", c_u64),
        ("model_params_alignment", c_u64), ("cost_params_size", c_u64),
        ("cost_params_alignment", c_u64), ("schema_hash", c_char_p), ("seed", c_u64),
    ]


class ProposalConfig(ctypes.Structure):
    """mppi_proposal_config (include/mppi_b200/mppi_proposal.h)."""
    _fields_ = [
        ("input_dim", c_u32), ("horizon", c_u32), ("control_dim", c_u32),
        ("max_batch", c_u32), ("seed", c_u64), ("log_scale_min", c_f32),
        ("log_scale_max", c_f32),
    ]


# name -> (restype, argtypes); every symbol the headers in include/mppi_b200 declare.
_ERR = [ctypes.c_char_p, c_size]
SIGNATURES = {
    # mppi_backend.h
    "mppi_backend_create": (ctypes.c_int, [ctypes.POINTER(c_ptr)]),
    "mppi_backend_destroy": (None, [c_ptr]),
    "mppi_backend_initialize": (ctypes.c_int, [c_ptr, ctypes.POINTER(BackendPlugin),
                                               ctypes.POINTER(BackendConfig)] + _ERR),
    "mppi_backend_bind_params": (ctypes.c_int, [c_ptr, c_ptr, c_size, c_ptr, c_size] + _ERR),
    "mppi_backend_dispatch_rollout": (ctypes.c_int, [c_ptr, c_u64, c_ptr, c_ptr, c_ptr, c_size,
                                                     c_ptr, c_size, c_ptr, c_ptr] + _ERR),
    "mppi_backend_dispatch_simulation": (ctypes.c_int, [c_ptr, c_u32, c_u64, c_ptr, c_ptr,
                                                        c_ptr, c_size, c_ptr, c_size, c_ptr,
                                                        c_ptr, c_ptr] + _ERR),
    "mppi_backend_dispatch_batch_simulation": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_u64, c_ptr,
                                                              c_ptr, ctypes.POINTER(BatchAgents),
                                                              c_ptr, c_ptr, c_ptr, c_ptr] + _ERR),
    "mppi_backend_reset": (ctypes.c_int, [c_ptr] + _ERR),
    "mppi_backend_batch_prepare": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr, c_ptr,
                                                  ctypes.POINTER(BatchAgents), c_u32, c_u32,
                                                  c_u32, c_u32] + _ERR),
    "mppi_backend_batch_run": (ctypes.c_int, [c_ptr, c_u64] + _ERR),
    "mppi_backend_last_run_ms": (ctypes.c_int, [c_ptr, ctypes.POINTER(c_f32)] + _ERR),
    "mppi_backend_batch_fetch": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr,
                                                c_ptr] + _ERR),
    "mppi_backend_last_costs": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_backend_last_cost_pairs": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_backend_last_weights": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_backend_sample_noise": (ctypes.c_int, [c_ptr, c_u64, c_u32, c_u32, c_u32, c_ptr,
                                                 c_ptr, c_ptr] + _ERR),
    "mppi_backend_time_passes": (ctypes.c_int, [c_ptr, c_u32, ctypes.POINTER(c_f32),
                                                ctypes.POINTER(c_f32)] + _ERR),
    "mppi_backend_launch_info": (ctypes.c_int, [c_ptr] + [ctypes.POINTER(c_u32)] * 5),
    "mppi_backend_step_form": (ctypes.c_int, [c_ptr, ctypes.POINTER(c_u32)]),
    "mppi_backend_tuning_info": (ctypes.c_int, [c_ptr] + [ctypes.POINTER(c_u32)] * 3
                                 + [ctypes.POINTER(c_f32)]),
    "mppi_device_philox": (ctypes.c_int, [c_u64, c_ptr, c_ptr, c_ptr, c_ptr] + _ERR),
    "mppi_device_sincos": (ctypes.c_int, [c_u64, c_ptr, ctypes.c_int, c_ptr, c_ptr] + _ERR),
    "mppi_device_log": (ctypes.c_int, [c_u64, c_ptr, c_ptr] + _ERR),
    "mppi_backend_dispatch_rollout_noalloc": (ctypes.c_int, [c_ptr, c_u64, c_ptr, c_ptr, c_ptr,
                                                             c_ptr, c_ptr, c_ptr] + _ERR),
    "mppi_backend_set_features": (ctypes.c_int, [c_ptr, ctypes.c_char_p, c_u32] + _ERR),
    "mppi_backend_features": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_backend_set_proposal": (ctypes.c_int, [c_ptr, c_ptr, c_u32] + _ERR),
    "mppi_backend_set_record_ustar": (ctypes.c_int, [c_ptr, c_u32] + _ERR),
    "mppi_backend_batch_fetch_ustar": (ctypes.c_int, [c_ptr, c_ptr] + _ERR),
    "mppi_backend_proposal_stage": (ctypes.c_int, [c_ptr, c_ptr, c_ptr, c_ptr] + _ERR),
    "mppi_backend_time_proposal": (ctypes.c_int, [c_ptr, c_u32, ctypes.POINTER(c_f32),
                                                  ctypes.POINTER(c_f32)] + _ERR),
    "mppi_compile_check": (ctypes.c_int, [ctypes.POINTER(BackendPlugin),
                                          ctypes.POINTER(BackendConfig), ctypes.c_char_p,
                                          c_size] + _ERR),
    "mppi_compile_check_proposal": (ctypes.c_int, [ctypes.POINTER(BackendPlugin),
                                                   ctypes.POINTER(BackendConfig), c_u32,
                                                   ctypes.c_char_p, ctypes.c_char_p, c_size]
                                    + _ERR),
    "mppi_b200_version": (ctypes.c_char_p, []),
    # mppi_proposal.h
    "mppi_proposal_create": (c_ptr, [ctypes.POINTER(ProposalConfig)] + _ERR),
    "mppi_proposal_destroy": (None, [c_ptr]),
    "mppi_proposal_param_count": (c_u64, [c_ptr]),
    "mppi_proposal_output_stride": (c_u32, [c_ptr]),
    "mppi_proposal_set_params": (ctypes.c_int, [c_ptr, c_ptr, c_u64] + _ERR),
    "mppi_proposal_get_params": (ctypes.c_int, [c_ptr, c_ptr, c_u64] + _ERR),
    "mppi_proposal_forward": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_proposal_gradients": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_ptr, c_u32, c_ptr, c_u32,
                                               ctypes.POINTER(c_f32), c_ptr] + _ERR),
    "mppi_proposal_train_step": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_ptr, c_u32, c_ptr, c_u32,
                                                c_f32, ctypes.POINTER(c_f32)] + _ERR),
    "mppi_proposal_last_train_ms": (c_f32, [c_ptr]),
    # mppi_driver_c.h
    "mppi_driver_create": (c_ptr, [ctypes.POINTER(DriverConfigC)]),
    "mppi_driver_destroy": (None, [c_ptr]),
    "mppi_driver_initialize": (ctypes.c_int, [c_ptr, ctypes.POINTER(DriverPluginC)] + _ERR),
    "mppi_driver_set_problem_params": (ctypes.c_int, [c_ptr, c_ptr, c_size, c_ptr, c_size] + _ERR),
    "mppi_driver_step": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_ptr, c_u32, c_u32, c_ptr, c_size,
                                        c_ptr, c_size, c_ptr, c_u32, c_u32, c_ptr] + _ERR),
    "mppi_driver_reset": (ctypes.c_int, [c_ptr] + _ERR),
    "mppi_driver_reset_nominal": (ctypes.c_int, [c_ptr, c_ptr, c_u32, c_u32] + _ERR),
    "mppi_driver_simulate": (ctypes.c_int, [c_ptr, c_u32, c_ptr, c_u32, c_ptr, c_u32, c_u32,
                                            c_ptr, c_size, c_ptr, c_size, c_ptr, c_ptr, c_ptr,
                                            c_u32] + _ERR),
    "mppi_driver_simulate_batch": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr, c_ptr, c_ptr,
                                                  c_ptr, c_ptr, c_u32, c_u32] + _ERR),
    "mppi_driver_simulate_batch_agents": (ctypes.c_int, [c_ptr, c_u32, c_u32, c_ptr, c_ptr,
                                                         c_size, c_ptr, c_size, c_ptr, c_ptr,
                                                         c_ptr, c_ptr, c_ptr, c_ptr, c_ptr,
                                                         c_u32, c_u32] + _ERR),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load libmppi_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("MPPI_B200_LIB", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -m mppi_metal_b200.build` "
            "(the library has no CPU or Python fallback)")
    lib = ctypes.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def err_buf(n: int = 8192):
    return ctypes.create_string_buffer(n)


def plugin_path(name: str) -> str:
    """Absolute path of a plugin source shipped in mppi_metal_b200/plugins."""
    p = PLUGIN_DIR / (name if name.endswith(".cu") else name + ".cu")
    return str(p)
