"""Every step form (plain or warp-specialised rollout, combine fused into the
rollout or a separate kernel) is its own compiled kernel, and the compiler may
contract a plugin's multiply-adds differently in each inlined copy of a
callable.  Results therefore stay independent of the (timed) form choice only
if the per-step state chain is the one rollout body, and the propagate and the
proposal features -- which the combine of every form computes -- are single
non-inlined functions.  Checked here on the kernel source (no GPU); the GPU
tests (test_gpu_fused_combine.py) compare the forms' results bit for bit."""
from __future__ import annotations

import re
from pathlib import Path

SRC = (Path(__file__).resolve().parents[1] / "mppi_metal_b200" / "csrc" / "device" /
       "mppi_kernels.cuh").read_text()


def _body(signature_regex: str) -> tuple[int, int]:
    """Span of the function definition (not a forward declaration)."""
    for m in re.finditer(signature_regex, SRC):
        brace, semi = SRC.find("{", m.end()), SRC.find(";", m.end())
        if brace != -1 and (semi == -1 or brace < semi):
            return m.start(), SRC.index("\n}\n", m.start())
    raise AssertionError(signature_regex)


def _calls(macro: str) -> list[int]:
    return [m.start() for m in re.finditer(re.escape(macro) + r"\(", SRC)]


def _inside(pos: int, span: tuple[int, int]) -> bool:
    return span[0] <= pos < span[1]


def test_feature_callable_has_one_compiled_copy():
    span = _body(r"__device__ __noinline__ void compute_features\(")
    calls = _calls("MPPI_FEATURES_FN")
    assert calls and all(_inside(p, span) for p in calls)
    assert len(_calls("compute_features")) >= 3  # definition, combine, features kernel


def test_propagate_has_one_compiled_copy():
    prop = _body(r"__device__ __noinline__ PropagateState propagate_dynamics\(")
    rollout = _body(r"__device__ __forceinline__ void rollout_item\(")
    calls = _calls("MPPI_DYNAMICS_FN")
    # the rollout's per-step recurrence and the propagate, nowhere else
    assert sum(_inside(p, prop) for p in calls) == 1
    assert sum(_inside(p, rollout) for p in calls) == 1
    assert len(calls) == 2
    combine = _body(r"__device__ __forceinline__ void combine_agent\(const MppiCombineArgs& a")
    assert any(_inside(p, combine) for p in _calls("propagate_dynamics"))
