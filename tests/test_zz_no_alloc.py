"""The allocation-free control step (mppi_backend_dispatch_rollout_noalloc).

It serves callers that may not allocate device memory while running -- a
fixed-rate robot control loop, where cudaMalloc / cudaFree can stall and
synchronise the device, or an application whose device memory belongs to
another allocator with a fixed budget.  Such a caller owns the input and
output buffers on the device; the step's temporary data lives in a static
device array inside the library.

The tests call the entry point through the C ABI on device buffers (made
with torch here, standing in for the caller's own) and check:
  * u_next and the diagnostics are the same bits as the regular entry point,
    mppi_backend_dispatch_rollout, for two calls in a row (the second one
    warm-started and at the next step index);
  * the same holds when the no-alloc step is the backend's first call, and
    right after the backend prepared a large batch (the step's launch shape
    is the single agent's whatever ran before);
  * a problem whose scratch exceeds the static array, and a backend with a
    learned proposal attached, are rejected with MPPI_ERR_INVALID and a
    message, before anything runs.
The file is collected last.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import backend_for
from mppi_metal_b200 import _lib, models
from mppi_metal_b200.backend import BackendError

pytestmark = pytest.mark.gpu


def _device(torch, a, dtype):
    return torch.as_tensor(np.array(a, copy=True), dtype=dtype).cuda().contiguous()


class _Buffers:
    """The caller's device buffers for one single-agent problem."""

    def __init__(self, torch, w, x0):
        self.torch = torch
        self.mp = _device(torch, np.frombuffer(w.model_params, np.uint8), torch.uint8)
        self.cp = _device(torch, np.frombuffer(w.cost_params[0], np.uint8), torch.uint8)
        self.x0 = _device(torch, x0, torch.float32)
        self.out = torch.zeros(w.horizon * w.control_dim, dtype=torch.float32, device="cuda")
        self.diag = torch.zeros(3, dtype=torch.float32, device="cuda")

    def step(self, b, step, u_nom):
        d_unom = _device(self.torch, u_nom, self.torch.float32)
        self.torch.cuda.synchronize()  # inputs complete before the call
        b.dispatch_rollout_noalloc(step, self.x0.data_ptr(), d_unom.data_ptr(),
                                   self.mp.data_ptr(), self.cp.data_ptr(), self.out.data_ptr(),
                                   self.diag.data_ptr())
        return self.out.cpu().numpy(), self.diag.cpu().numpy()


def _two_steps_match(torch, w, b_noalloc, b_ref, x0):
    buf = _Buffers(torch, w, x0)
    u_nom = np.zeros(w.horizon * w.control_dim, np.float32)
    for step in (0, 1):
        u, diag = buf.step(b_noalloc, step, u_nom)
        ref_u, ref_diag = b_ref.dispatch_rollout(step, x0, u_nom)
        assert np.array_equal(u, ref_u), np.max(np.abs(u - ref_u))
        assert np.array_equal(diag, ref_diag), (diag, ref_diag)
        # next call: warm start (shift left, hold last), as MPPIDriver::step does
        u_nom = np.concatenate([ref_u[w.control_dim:], ref_u[-w.control_dim:]])


def test_noalloc_step_matches_dispatch_rollout_twice():
    torch = pytest.importorskip("torch")
    w = models.unicycle_single(seed=3, K=1024, H=30)
    b = backend_for(w)  # binds the same blobs the no-alloc call receives by pointer
    x0 = np.array([0.5, -1.0, 0.2, 0.0], np.float32)
    _two_steps_match(torch, w, b, b, x0)


def test_noalloc_step_first_call_and_after_large_batch():
    torch = pytest.importorskip("torch")
    w = models.unicycle_single(seed=5, K=4096, H=30)
    x0 = np.array([-2.0, 1.0, 0.7, 0.0], np.float32)
    ref = backend_for(w)
    fresh = backend_for(w)  # the no-alloc step is this backend's first call
    _two_steps_match(torch, w, fresh, ref, x0)
    # a prepared batch of many agents on the same backend changes the batch
    # launch shape, not the single agent's
    wb = models.unicycle_batch(seed=9, N=64, K=4096, H=30, T=2)
    fresh.prepare(wb.num_agents, 2, wb.x0, cost_params=wb.cost_params_packed,
                  cost_stride=wb.cost_stride, sigma=wb.agent_sigma)
    fresh.run(0)
    _two_steps_match(torch, w, fresh, ref, x0)


def test_noalloc_step_rejects_oversized_problem():
    torch = pytest.importorskip("torch")
    # 2^20 samples: 8192 rollout blocks of (8 + 60) floats of partial sums,
    # more than the static array holds
    w = models.unicycle_single(seed=0, K=1 << 20, H=30)
    b = backend_for(w)
    buf = _Buffers(torch, w, np.zeros(4, np.float32))
    with pytest.raises(BackendError) as e:
        buf.step(b, 0, np.zeros(w.horizon * w.control_dim, np.float32))
    assert e.value.code == _lib.MPPI_ERR_INVALID
    assert "bytes of scratch" in e.value.msg
    assert not torch.any(buf.out != 0).item()  # nothing ran


def test_noalloc_step_rejects_attached_proposal():
    torch = pytest.importorskip("torch")
    from mppi_metal_b200 import proposal as P
    w = models.unicycle_single(seed=1, K=1024, H=30)
    b = backend_for(w)
    net = P.ProposalNet(P.UNICYCLE_FEATURES, w.horizon, w.control_dim, max_batch=128, seed=0)
    b.set_features(P.FEATURES_CALLABLE, P.UNICYCLE_FEATURES)
    b.set_proposal(net, 256)
    buf = _Buffers(torch, w, np.zeros(4, np.float32))
    with pytest.raises(BackendError) as e:
        buf.step(b, 0, np.zeros(w.horizon * w.control_dim, np.float32))
    assert e.value.code == _lib.MPPI_ERR_INVALID
    assert "proposal" in e.value.msg
    # detached, the backend runs the no-alloc step again, with the bits of
    # its own regular step
    b.set_proposal(None)
    _two_steps_match(torch, w, b, b, np.zeros(4, np.float32))
