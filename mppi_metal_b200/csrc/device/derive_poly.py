"""Derives the polynomial coefficients of the library's own sine / cosine
and natural logarithm (mppi_prelude.cuh: mppi_sincos_quarter, mppi_sincosf,
mppi_log) and checks the error of the float32 evaluation the device performs.

    python mppi_metal_b200/csrc/device/derive_poly.py

Method: near-minimax polynomials by Lawson's iteratively reweighted least
squares on a dense grid (C. L. Lawson, "Contributions to the theory of
linear least maximum approximation", 1961), fitted in float64 to the
relative error of sin and the absolute error of cos, then rounded to float32.
The printed errors come from evaluating the rounded coefficients the way the
device does (float32 FMA Horner steps, emulated exactly through float64
products) against numpy's float64 sin / cos.

Three families:
  logarithm:     ln x = e ln 2 + f + f^2 * P(f), x = 2^e (1 + f), f in [-1/3, 1/3)
                 (the exponent is split off around 2/3 so that f is exact)
  quarter-turn:  s(f) = sin(pi/2 f) = f * S(f^2),  c(f) = cos(pi/2 f) = C(f^2)
                 for f in [-1/2, 1/2] (Box-Muller's angle 2 pi u = pi/2 (q + f))
  radians:       sin(r) = r + r^3 * S(r^2),  cos(r) = 1 + r^2 * C(r^2)
                 for r in [-pi/4, pi/4] (after the Cody-Waite reduction by pi/2)
"""
from __future__ import annotations

import numpy as np


def lawson(basis: np.ndarray, target: np.ndarray, weight: np.ndarray, iters: int = 400):
    """Weighted minimax fit: minimise max |weight * (basis @ c - target)|."""
    A = basis * weight[:, None]
    b = target * weight
    w = np.full(len(b), 1.0 / len(b))
    c = None
    for _ in range(iters):
        sw = np.sqrt(w)
        c, *_ = np.linalg.lstsq(A * sw[:, None], b * sw, rcond=None)
        e = np.abs(A @ c - b)
        w = w * e
        s = w.sum()
        if s == 0:
            break
        w /= s
    return c


def f32(x):
    return np.float32(x)


def fma32(a, b, c):
    """float32 fused multiply-add: the float32 product is exact in float64."""
    return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)


def horner32(coefs, z):
    """c[0] + z (c[1] + z (c[2] + ...)) with float32 FMA steps."""
    acc = np.full_like(z, coefs[-1], dtype=np.float32)
    for cf in coefs[-2::-1]:
        acc = fma32(acc, z, np.float32(cf))
    return acc


def hexf(x: np.float32) -> str:
    """C hexadecimal float literal of a float32 value (exact)."""
    h = float(x).hex()  # e.g. '-0x1.921fb60000000p+0'
    mant, exp = h.split("p")
    mant = mant.rstrip("0").rstrip(".")
    return f"{mant}p{exp}f"


def fit_quarter():
    f = np.linspace(1e-6, 0.5, 200001)
    z = f * f
    # sin(pi/2 f) / f = S(z), degree 3 in z (f, f^3, f^5, f^7); relative error
    B = np.stack([z ** i for i in range(4)], axis=1)
    ts = np.sin(np.pi / 2 * f) / f
    cs = lawson(B, ts, 1.0 / ts)
    # cos(pi/2 f) = 1 + z * C(z), degree 3 in z (z .. z^4); absolute error
    Bc = np.stack([z ** (i + 1) for i in range(4)], axis=1)
    cc = lawson(Bc, np.cos(np.pi / 2 * f) - 1.0, np.ones_like(f))
    return [f32(x) for x in cs], [f32(x) for x in cc]


def fit_radians():
    r = np.linspace(1e-6, np.pi / 4, 200001)
    z = r * r
    # (sin r - r) / r^3 = S(z), degree 2 in z (r^3, r^5, r^7)... relative to sin
    B = np.stack([z ** i for i in range(3)], axis=1)
    ts = (np.sin(r) - r) / (r ** 3)
    ws = r ** 3 / np.sin(r)
    cs = lawson(B, ts, ws)
    # (cos r - 1) / r^2 = C(z), degree 3 in z (r^2 .. r^8); absolute error
    Bc = np.stack([z ** i for i in range(4)], axis=1)
    tc = (np.cos(r) - 1.0) / z
    cc = lawson(Bc, tc, z)
    return [f32(x) for x in cs], [f32(x) for x in cc]


def fit_log(deg: int = 7):
    """(ln(1 + f) - f) / f^2 = P(f) on [-1/3, 1/3]; weighted to the relative
    error of ln(1 + f)."""
    f = np.concatenate([np.linspace(-1.0 / 3.0, -1e-5, 200001), np.linspace(1e-5, 1.0 / 3.0, 200001)])
    B = np.stack([f ** i for i in range(deg + 1)], axis=1)
    t = (np.log1p(f) - f) / (f * f)
    w = (f * f) / np.abs(np.log1p(f))
    return [f32(x) for x in lawson(B, t, w)]


LN2_HI = f32(0.693145751953125)          # 0x1.62e4p-1: 11 significant bits, e * LN2_HI exact
LN2_LO = f32(np.log(2.0) - 0.693145751953125)


def log32(x, c):
    """The device's float32 evaluation of ln x for normal x > 0."""
    i = x.view(np.int32).astype(np.int64)
    e = (i - 0x3F2AAAAB) >> 23
    m = (i - (e << 23)).astype(np.int32).view(np.float32)
    f = (m - np.float32(1.0)).astype(np.float32)
    z = (f * f).astype(np.float32)
    p = horner32(c, f)
    r = fma32(p, z, f)
    ef = e.astype(np.float32)
    return fma32(ef, LN2_HI, fma32(ef, LN2_LO, r))


def check_log(c):
    rng = np.random.default_rng(0)
    u = np.concatenate([
        ((rng.integers(0, 2 ** 32, 2000000, dtype=np.uint64).astype(np.float32) + np.float32(0.5))
         * np.float32(2.0 ** -32)).astype(np.float32),
        np.float32(1.0) - np.arange(1, 20000, dtype=np.float32) * np.float32(2.0 ** -24),
        np.float32(2.0) ** -np.arange(1, 33, dtype=np.float32)])
    got = log32(u, c).astype(np.float64)
    ref = np.log(u.astype(np.float64))
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-30)
    return rel.max(), np.abs(got - ref).max()


def check_quarter(cs, cc):
    f = np.linspace(-0.5, 0.5, 2000001).astype(np.float32)
    z = (f * f).astype(np.float32)
    s = (f * horner32(cs, z)).astype(np.float32)
    c = fma32(horner32(cc, z), z, np.float32(1.0))
    es = np.abs(s.astype(np.float64) - np.sin(np.pi / 2 * f.astype(np.float64)))
    ec = np.abs(c.astype(np.float64) - np.cos(np.pi / 2 * f.astype(np.float64)))
    return es.max(), ec.max()


def check_radians(cs, cc):
    r = np.linspace(-np.pi / 4, np.pi / 4, 2000001).astype(np.float32)
    z = (r * r).astype(np.float32)
    r3 = (r * z).astype(np.float32)
    s = fma32(horner32(cs, z), r3, r)
    c = fma32(horner32(cc, z), z, np.float32(1.0))
    rd = r.astype(np.float64)
    es = np.abs(s.astype(np.float64) - np.sin(rd))
    ec = np.abs(c.astype(np.float64) - np.cos(rd))
    return es.max(), ec.max()


def main():
    qs, qc = fit_quarter()
    rs, rc = fit_radians()
    print("quarter-turn sin S(z):", ", ".join(hexf(x) for x in qs))
    print("quarter-turn cos C(z):", ", ".join(hexf(x) for x in qc))
    print("  max abs error (float32 evaluation): sin %.3g  cos %.3g" % check_quarter(qs, qc))
    print("radians sin S(z):", ", ".join(hexf(x) for x in rs))
    print("radians cos C(z):", ", ".join(hexf(x) for x in rc))
    print("  max abs error on [-pi/4, pi/4] (float32 evaluation): sin %.3g  cos %.3g"
          % check_radians(rs, rc))
    lc = fit_log()
    print("log P(f):", ", ".join(hexf(x) for x in lc))
    print("  max error of ln u on u = (x + 0.5) 2^-32 (float32 evaluation): rel %.3g  abs %.3g"
          % check_log(lc))
    print("ln2 split:", hexf(LN2_HI), hexf(LN2_LO))
    # Cody-Waite split of pi/2 for the FMA reduction r = x - q (C1 + C2 + C3)
    c1 = f32(np.pi / 2)
    c2 = f32(np.pi / 2 - np.float64(c1))
    c3 = f32(np.pi / 2 - np.float64(c1) - np.float64(c2))
    print("pi/2 split:", hexf(c1), hexf(c2), hexf(c3))


if __name__ == "__main__":
    main()
