"""The proposal network's CPU restatement (oracle/mlp_oracle.py), pinned
without a GPU: bfloat16 rounding on known values, and the analytic gradient
of the float64 network against central finite differences."""
from __future__ import annotations

import numpy as np

import mlp_oracle as mo


def test_bf16_rounding_known_values():
    one = 1.0
    ulp = 2.0 ** -7                      # bf16 spacing in [1, 2)
    vals = np.array([one, one + ulp / 2, one + 3 * ulp / 2, one + ulp / 4, -2.5, 3.0e-39])
    got = mo.bf16(vals)
    # ties to even: 1 + ulp/2 -> 1, 1 + 3ulp/2 -> 1 + 2ulp; 1 + ulp/4 -> 1
    assert got[0] == 1.0 and got[1] == 1.0 and got[2] == one + 2 * ulp and got[3] == 1.0
    assert got[4] == -2.5
    assert np.isfinite(got[5])


def test_shape_and_param_layout():
    s = mo.Shape(31, 64, 2)
    assert s.hm == 128 and s.out_dim == 130 and s.out_pad == 144
    assert s.param_count == 256 * 32 + 256 + 2 * (256 * 256 + 256) + 144 * 256 + 144
    p = mo.init_params(s, 0)
    (W0, _), _, _, (W3, b3) = mo.unpack(s, p)
    assert np.all(W0[:, 31:] == 0) and np.all(W3[130:] == 0) and np.all(b3[130:] == 0)
    assert np.array_equal(mo.pack(mo.unpack(s, p)), p.astype(np.float64))


def test_gradient_matches_finite_differences():
    s = mo.Shape(7, 5, 2, log_scale_min=-3.0, log_scale_max=1.0)
    rng = np.random.default_rng(1)
    p = mo.init_params(s, 3).astype(np.float64)
    x = rng.normal(size=(6, 7))
    y = rng.normal(size=(6, s.hm)) * 0.5
    loss, g = mo.loss_and_grad(s, p, x, y, mirror=False)
    assert np.isfinite(loss)
    # a sample of live parameters from every layer (weights and biases)
    layers = mo.unpack(s, np.arange(s.param_count, dtype=np.float64))
    idx = []
    for l, (W, b) in enumerate(layers):
        rows = s.out_dim if l == 3 else W.shape[0]
        cols = s.input_dim if l == 0 else W.shape[1]
        for _ in range(6):
            idx.append(int(W[rng.integers(rows), rng.integers(cols)]))
        idx.append(int(b[rng.integers(rows)]))
    # the log-scale outputs' biases (the NLL's variance path)
    idx += [int(layers[3][1][s.hm]), int(layers[3][1][s.hm + 1])]
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_and_grad(s, pp, x, y, mirror=False)[0]
              - mo.loss_and_grad(s, pm, x, y, mirror=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_mirrored_rounding_stays_close_to_float64():
    s = mo.Shape(31, 64, 2)
    rng = np.random.default_rng(2)
    p = mo.init_params(s, 5).astype(np.float64)
    x = rng.normal(size=(64, 31))
    y = rng.normal(size=(64, s.hm))
    l64, g64 = mo.loss_and_grad(s, p, x, y, mirror=False)
    l16, g16 = mo.loss_and_grad(s, p, x, y, mirror=True)
    assert abs(l16 - l64) < 1e-2 * abs(l64)
    assert np.linalg.norm(g16 - g64) < 3e-2 * np.linalg.norm(g64)
