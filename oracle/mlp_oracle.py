"""CPU restatement of the learned-proposal network (numpy, float64).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the tcgen05 kernels of
mppi_metal_b200/csrc/proposal_mlp.cu; the product never imports it.

The network has no reference counterpart (the reference samples only around
the warm start, shaders/mppi_rollout.metal:96-112), so this file restates the
method as include/mppi_b200/mppi_proposal.h defines it:

  in (<= 32, zero-padded to 32) -> 256 -> 256 -> 256 -> P   (P = round16(H m + m))
  hidden: h = GELU(z), z = W x + b, exact-erf GELU
  loss  : mean over rows and the H m entries of 0.5 (u* - mu)^2 exp(-2 c_d) + c_d,
          c_d = clip(s_d, lo, hi), s = out[H m : H m + m]

`mirror=True` rounds to bfloat16 exactly where the kernels do (inputs,
weights, hidden activations, and every gradient that feeds a tensor-core
GEMM); `mirror=False` is the plain float64 network, pinned by central finite
differences in tests/test_proposal_oracle.py.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

HID = 256
IN_PAD = 32


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (round to nearest even, via float32), as float64."""
    f = np.ascontiguousarray(np.asarray(x, np.float64).astype(np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


@dataclass
class Shape:
    input_dim: int
    horizon: int
    control_dim: int
    log_scale_min: float = -3.0
    log_scale_max: float = 1.0

    @property
    def hm(self) -> int:
        return self.horizon * self.control_dim

    @property
    def out_dim(self) -> int:
        return self.hm + self.control_dim

    @property
    def out_pad(self) -> int:
        return (self.out_dim + 15) // 16 * 16

    def layer_dims(self):
        """(rows, cols) of W0..W3."""
        return [(HID, IN_PAD), (HID, HID), (HID, HID), (self.out_pad, HID)]

    @property
    def param_count(self) -> int:
        return sum(r * c + r for r, c in self.layer_dims())


def unpack(shape: Shape, flat: np.ndarray):
    """Flat parameter vector -> [(W, b)] (the order of mppi_proposal.h)."""
    out, o = [], 0
    for r, c in shape.layer_dims():
        W = np.asarray(flat[o:o + r * c], np.float64).reshape(r, c)
        o += r * c
        b = np.asarray(flat[o:o + r], np.float64)
        o += r
        out.append((W, b))
    assert o == len(flat)
    return out


def pack(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b]) for W, b in layers])


def init_params(shape: Shape, seed: int) -> np.ndarray:
    """Random parameters with the padding entries zero (for tests)."""
    rng = np.random.default_rng(seed)
    layers = []
    for l, (r, c) in enumerate(shape.layer_dims()):
        fan_in = shape.input_dim if l == 0 else HID
        bound = 1.0 / math.sqrt(fan_in) * (0.3 if l == 3 else 1.0)
        W = np.zeros((r, c))
        b = np.zeros(r)
        rows = shape.out_dim if l == 3 else r
        W[:rows, :fan_in] = rng.uniform(-bound, bound, (rows, fan_in))
        b[:rows] = rng.uniform(-bound, bound, rows)
        layers.append((W, b))
    return pack(layers).astype(np.float32)


def forward(shape: Shape, flat, x, mirror=True, keep=False):
    """Network outputs [M][out_pad] (and the intermediates when keep)."""
    rnd = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    layers = unpack(shape, flat)
    M = x.shape[0]
    xin = np.zeros((M, IN_PAD))
    xin[:, :shape.input_dim] = np.asarray(x, np.float64)[:, :shape.input_dim]
    h = [rnd(xin)]
    zs = []
    for l in range(3):
        W, b = layers[l]
        z = h[-1] @ rnd(W).T + b
        zs.append(z)
        h.append(rnd(gelu(z)))
    W, b = layers[3]
    out = h[-1] @ rnd(W).T + b
    if keep:
        return out, zs, h
    return out


def loss_and_grad(shape: Shape, flat, x, target, mirror=True):
    """(loss, flat gradient) of the proposal loss over all rows of x."""
    rnd = bf16 if mirror else (lambda a: np.asarray(a, np.float64))
    layers = unpack(shape, flat)
    out, zs, h = forward(shape, flat, x, mirror=mirror, keep=True)
    M, hm, m = x.shape[0], shape.hm, shape.control_dim
    inv_norm = 1.0 / (M * hm)
    mu = out[:, :hm].reshape(M, shape.horizon, m)
    raw = out[:, hm:hm + m]
    c = np.clip(raw, shape.log_scale_min, shape.log_scale_max)
    inside = (raw > shape.log_scale_min) & (raw < shape.log_scale_max)
    iv = np.exp(-2.0 * c)                                       # [M][m]
    diff = np.asarray(target, np.float64)[:, :hm].reshape(M, shape.horizon, m) - mu
    loss = inv_norm * float(np.sum(0.5 * diff ** 2 * iv[:, None, :] + c[:, None, :]))
    dmu = -diff * iv[:, None, :] * inv_norm
    dc = np.sum(1.0 - diff ** 2 * iv[:, None, :], axis=1) * inv_norm
    dout = np.zeros((M, shape.out_pad))
    dout[:, :hm] = dmu.reshape(M, hm)
    dout[:, hm:hm + m] = dc * inside
    dz = [None, None, None, rnd(dout)]
    for l in (3, 2, 1):
        W, _ = layers[l]
        dh = dz[l] @ rnd(W)
        dz[l - 1] = rnd(dh * gelu_grad(zs[l - 1]))
    grads = [(dz[l].T @ h[l], dz[l].sum(axis=0)) for l in range(4)]
    return loss, pack(grads)


def adam(flat, grad, m1, m2, t, lr, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (bias correction folded into the step size, as the kernel does)."""
    m1 = beta1 * m1 + (1 - beta1) * grad
    m2 = beta2 * m2 + (1 - beta2) * grad * grad
    lr_t = lr * math.sqrt(1 - beta2 ** t) / (1 - beta1 ** t)
    return flat - lr_t * m1 / (np.sqrt(m2) + eps), m1, m2


# ---------------------------------------------------------------------------
# Proposal features of the unicycle plugin (mppi_proposal_features in
# mppi_metal_b200/plugins/unicycle_obstacles.cu; blob layout in
# plugins/model_params.h: 8 header words, then cx, cy, vx, vy, r x 16).
# ---------------------------------------------------------------------------
UNICYCLE_MAX_OBS = 16


def unicycle_cost_fields(blob: bytes):
    w = np.frombuffer(blob, dtype=np.float32)
    n = int(np.frombuffer(blob[20:24], dtype=np.uint32)[0])
    obs = w[8:8 + 5 * UNICYCLE_MAX_OBS].astype(np.float64).reshape(5, UNICYCLE_MAX_OBS)
    return float(w[0]), float(w[1]), min(n, UNICYCLE_MAX_OBS), obs


def unicycle_features(state, blob: bytes) -> np.ndarray:
    """The 31 features of one state [x, y, theta, t] (float64)."""
    gx, gy, n, (cx, cy, vx, vy, r) = unicycle_cost_fields(blob)
    x, y, th, t = (float(v) for v in state[:4])
    cs, sn = math.cos(th), math.sin(th)
    f = np.zeros(31)
    f[:5] = [x * 0.1, y * 0.1, cs, sn, t / 15.0]
    dx, dy = gx - x, gy - y
    f[5] = (cs * dx + sn * dy) * 0.1
    f[6] = (cs * dy - sn * dx) * 0.1
    ex = cx[:n] + vx[:n] * t - x
    ey = cy[:n] + vy[:n] * t - y
    clr = np.sqrt(ex * ex + ey * ey) - r[:n]
    order = np.argsort(clr, kind="stable")[:8]
    for j, i in enumerate(order):
        f[7 + 3 * j] = (cs * ex[i] + sn * ey[i]) * 0.1
        f[8 + 3 * j] = (cs * ey[i] - sn * ex[i]) * 0.1
        f[9 + 3 * j] = r[i]
    return f


# Proposal features of the quadrotor plugin (mppi_proposal_features in
# mppi_metal_b200/plugins/quadrotor.cu; QuadrotorCostParams: 12 header words,
# then cx, cy, cz, r x 32).
QUAD_MAX_OBS = 32


def quadrotor_features(state, blob: bytes) -> np.ndarray:
    """The 29 features of one quadrotor state (float64)."""
    w = np.frombuffer(blob, dtype=np.float32).astype(np.float64)
    n = min(int(np.frombuffer(blob[36:40], dtype=np.uint32)[0]), QUAD_MAX_OBS)
    wp = w[0:3]
    cx, cy, cz, r = w[12:12 + 4 * QUAD_MAX_OBS].reshape(4, QUAD_MAX_OBS)
    s = np.asarray(state, np.float64)
    f = np.zeros(29)
    f[0:3] = (s[0:3] - wp) * 0.25
    f[3:6] = s[3:6] * 0.5
    f[6:9] = s[6:9]
    f[9:12] = s[9:12] * 0.25
    f[12] = s[2] * 0.25
    ex, ey, ez = cx[:n] - s[0], cy[:n] - s[1], cz[:n] - s[2]
    clr = np.sqrt(ex * ex + ey * ey + ez * ez) - r[:n]
    for j, i in enumerate(np.argsort(clr, kind="stable")[:4]):
        f[13 + 4 * j:17 + 4 * j] = [ex[i] * 0.25, ey[i] * 0.25, ez[i] * 0.25, r[i]]
    return f
