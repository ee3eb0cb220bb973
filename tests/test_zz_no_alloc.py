"""The allocation-free control step (mppi_backend_dispatch_rollout_noalloc).

It serves callers that may not allocate device memory while running -- a
fixed-rate robot control loop, where cudaMalloc / cudaFree can stall and
synchronise the device, or an application whose device memory belongs to
another allocator with a fixed budget.  Such a caller owns the input and
output buffers on the device; the step's temporary data lives in a static
device array inside the library.

The test calls the entry point through the C ABI on device buffers (made
with torch here, standing in for the caller's own) and checks its u_next and
diagnostics against the regular entry point, mppi_backend_dispatch_rollout,
for two calls in a row (the second one warm-started and at the next step
index), within the u_next tolerance of the parity tests.  It sits in a file
of its own, collected last.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import backend_for
from mppi_metal_b200 import models

pytestmark = pytest.mark.gpu

TOL_U = 1e-4


def _device(torch, a, dtype):
    return torch.as_tensor(np.array(a, copy=True), dtype=dtype).cuda().contiguous()


def test_noalloc_step_matches_dispatch_rollout_twice():
    torch = pytest.importorskip("torch")
    w = models.unicycle_single(seed=3, K=1024, H=30)
    b = backend_for(w)  # binds the same blobs the no-alloc call receives by pointer
    x0 = np.array([0.5, -1.0, 0.2, 0.0], np.float32)
    u_nom = np.zeros(w.horizon * w.control_dim, np.float32)

    d_mp = _device(torch, np.frombuffer(w.model_params, np.uint8), torch.uint8)
    d_cp = _device(torch, np.frombuffer(w.cost_params[0], np.uint8), torch.uint8)
    d_x0 = _device(torch, x0, torch.float32)
    d_out = torch.zeros(w.horizon * w.control_dim, dtype=torch.float32, device="cuda")
    d_diag = torch.zeros(3, dtype=torch.float32, device="cuda")

    for step in (0, 1):
        ref_u, ref_diag = b.dispatch_rollout(step, x0, u_nom)
        d_unom = _device(torch, u_nom, torch.float32)
        torch.cuda.synchronize()
        b.dispatch_rollout_noalloc(step, d_x0.data_ptr(), d_unom.data_ptr(), d_mp.data_ptr(),
                                   d_cp.data_ptr(), d_out.data_ptr(), d_diag.data_ptr())
        u = d_out.cpu().numpy()
        diag = d_diag.cpu().numpy()
        assert np.max(np.abs(u - ref_u)) <= TOL_U
        assert np.max(np.abs(diag - ref_diag) / np.maximum(np.abs(ref_diag), 1.0)) <= 1e-5
        # next call: warm start (shift left, hold last), as MPPIDriver::step does
        u_nom = np.concatenate([ref_u[w.control_dim:], ref_u[-w.control_dim:]])
