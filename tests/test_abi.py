"""The C ABI boundary, without a GPU: the library loads, exports every
function the public headers declare, and every shipped plugin compiles with
the library kernels for sm_100a through NVRTC."""
from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

from mppi_metal_b200 import _lib
from mppi_metal_b200.backend import compile_check

INCLUDE = Path(_lib.INCLUDE_DIR)


def declared_c_functions() -> set[str]:
    names = set()
    for h in (INCLUDE / "mppi_b200").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mppi_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_loads(lib):
    assert b"sm_100a" in lib.mppi_b200_version()


def test_every_declared_symbol_is_exported(lib):
    names = declared_c_functions()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_the_headers():
    assert declared_c_functions() == set(_lib.SIGNATURES)


def test_cpp_driver_symbols_exported(lib):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", str(_lib.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    for sym in ["mppi_metal::MPPIDriver::MPPIDriver(mppi_metal::DriverConfig const&)",
                "mppi_metal::MPPIDriver::initialize(",
                "mppi_metal::MPPIDriver::set_problem_params(",
                "mppi_metal::MPPIDriver::step(",
                "mppi_metal::MPPIDriver::reset(std::",
                "mppi_metal::MPPIDriver::reset(mppi_metal::ControlSequenceView const&",
                "mppi_metal::MPPIDriver::simulate(",
                "mppi_metal::MPPIDriver::simulate_batch("]:
        assert sym in out, sym


PLUGINS = [
    ("double_integrator", 4, 2, 0, 0),
    ("nonholonomic_vehicle", 4, 2, 8, 24),
    ("unicycle_obstacles", 4, 2, 16, 352),
    ("gust_integrator", 5, 2, 16, 0),
    ("bicycle_lane", 5, 2, 16, 544),
    ("quadrotor", 12, 4, 32, 560),
    ("wez_environment", 45, 2, 40, 32),  # 180-byte state: beyond the reference's 128
]


@pytest.mark.parametrize("plugin,n,m,mp,cp", PLUGINS)
@pytest.mark.parametrize("cov_full,control_cost", [(False, False), (True, True)])
def test_plugins_compile_for_sm100a(plugin, n, m, mp, cp, cov_full, control_cost):
    rc, err, log = compile_check(plugin, n, m, cov_full=cov_full, control_cost=control_cost,
                                 model_params_size=mp, cost_params_size=cp)
    assert rc == 0, err
    assert "mppi_rollout_b128" in log and "sm_100a" in log
    # no register spills in the benchmark model's hot kernel
    block = log.split("Function properties for mppi_rollout_b128")[1].split("Compile time")[0]
    if plugin == "unicycle_obstacles":
        assert "0 bytes spill stores" in block


def test_missing_callable_is_named():
    rc, err, _ = compile_check("double_integrator", 4, 2, dynamics="nonexistent_fn")
    assert rc == _lib.MPPI_ERR_CALLABLE
    assert "nonexistent_fn" in err


def test_missing_cost_callable_is_named():
    rc, err, _ = compile_check("double_integrator", 4, 2, stage_cost="no_such_cost")
    assert rc == _lib.MPPI_ERR_CALLABLE
    assert "no_such_cost" in err


def test_unreadable_plugin_is_reported():
    rc, err, _ = compile_check("/nonexistent/plugin.cu", 4, 2)
    assert rc == _lib.MPPI_ERR_PLUGIN
    assert "/nonexistent/plugin.cu" in err


def test_plugin_compile_error_is_reported(tmp_path):
    bad = tmp_path / "bad.cu"
    bad.write_text('#include "mppi_core.h"\n__device__ void mppi_dynamics(uint8_t* s, '
                   'const float* u, const uint8_t* p, uint2 c, uint32_t k) { this is not C++ }\n')
    rc, err, _ = compile_check(str(bad), 4, 2, stage_cost="", terminal_cost="")
    assert rc == _lib.MPPI_ERR_PLUGIN
    assert "bad.cu" in err


def test_reference_style_plugin_includes_resolve(tmp_path):
    """A plugin written like the reference's (includes "mppi_core.h" and
    "philox.h", declares state as uint8_t*, draws Philox numbers in its
    dynamics) compiles unchanged apart from the address-space keywords."""
    src = tmp_path / "stochastic.cu"
    src.write_text(
        '#include "mppi_core.h"\n#include "philox.h"\n'
        "__device__ void mppi_dynamics(uint8_t* state_raw, const float* control,\n"
        "    const uint8_t* mp, uint2 rng_counter, uint32_t rng_seed) {\n"
        "  float* s = (float*)state_raw;\n"
        "  uint2 c = make_uint2(rng_counter.x, rng_counter.y + 0x1000u);\n"
        "  float u = uint_to_01(philox2x32_10(c, rng_seed).x);\n"
        "  s[0] += 0.1f * control[0] + 0.01f * u;\n"
        "  s[1] += 0.1f * control[1];\n}\n")
    rc, err, _ = compile_check(str(src), 2, 2, stage_cost="", terminal_cost="")
    assert rc == 0, err


def test_queries_before_initialize_report_not_init(lib):
    """A created backend answers the measurement queries with
    MPPI_ERR_NOT_INIT until initialize (no device call is made)."""
    import ctypes
    h = ctypes.c_void_p()
    assert lib.mppi_backend_create(ctypes.byref(h)) == 0
    try:
        form = ctypes.c_uint32(99)
        assert lib.mppi_backend_step_form(h, ctypes.byref(form)) == _lib.MPPI_ERR_NOT_INIT
        assert form.value == 99
        vals = [ctypes.c_uint32() for _ in range(5)]
        assert lib.mppi_backend_launch_info(h, *[ctypes.byref(v) for v in vals]) == \
            _lib.MPPI_ERR_NOT_INIT
        assert lib.mppi_backend_step_form(None, ctypes.byref(form)) == _lib.MPPI_ERR_NOT_INIT
    finally:
        lib.mppi_backend_destroy(h)


# ---- ParamLayout against a plugin's declared layout (MPPI_PARAM_LAYOUT) ----
# The reference declares ParamLayout::schema_hash and alignments
# (include/mppi_metal/mppi_types.hpp:88-94) and its README promises that
# initialize fails when the declared layout does not match the binding; the
# shipped plugins declare theirs, and the module compile checks them.

def _layout_check(**kw):
    base = dict(model_params_size=16, cost_params_size=352)
    base.update(kw)
    return compile_check("unicycle_obstacles", 4, 2, **base)


def test_declared_layout_accepts_matching_param_layout():
    for kw in ({}, dict(model_params_alignment=4, cost_params_alignment=16),
               dict(schema_hash="mppi_b200/unicycle_obstacles/1")):
        rc, err, _ = _layout_check(**kw)
        assert rc == 0, (kw, err)


@pytest.mark.parametrize("kw,field", [
    (dict(model_params_size=20), "ParamLayout::model_params_size"),
    (dict(cost_params_size=348), "ParamLayout::cost_params_size"),
    (dict(model_params_alignment=2), "ParamLayout::model_params_alignment"),
    (dict(cost_params_alignment=2), "ParamLayout::cost_params_alignment"),
    (dict(schema_hash="mppi_b200/unicycle_obstacles/2"), "ParamLayout::schema_hash"),
])
def test_declared_layout_mismatch_is_named(kw, field):
    rc, err, _ = _layout_check(**kw)
    assert rc == _lib.MPPI_ERR_INVALID, err
    assert field in err and "does not match" in err, err


def test_schema_hash_characters_are_checked():
    rc, err, _ = _layout_check(schema_hash='bad"quote')
    assert rc == _lib.MPPI_ERR_INVALID
    assert "schema_hash" in err


def test_undeclared_plugin_keeps_reference_binding():
    # the reference's own test plugin declares no layout: any sizes, any
    # schema string compile (the reference checks sizes against blobs only)
    rc, err, _ = compile_check("double_integrator", 4, 2, model_params_size=16,
                               cost_params_size=8, schema_hash="anything")
    assert rc == 0, err


def test_state_limit_is_named():
    # the state buffer is sized per module up to MPPI_MAX_STATE_DIM floats;
    # beyond it initialize fails naming state_dim (validation, no GPU)
    from mppi_metal_b200 import driver as D
    s = np.ones(2, np.float32)
    cfg = D.DriverConfig(state_dim=129, control_dim=2, horizon=10, sample_count=64,
                         noise=D.ControlNoiseConfig(D.CovarianceForm.kDiagonal, s, s, 2),
                         bounds=D.ControlBounds(-s, s, 2))
    drv = D.MPPIDriver(cfg)
    err = D.ErrorRef()
    assert not drv.initialize(D.ModelPluginSpec(_lib.plugin_path("double_integrator")), err)
    assert "state_dim" in err.value and "128 floats" in err.value, err.value
