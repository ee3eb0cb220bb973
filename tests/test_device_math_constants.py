"""The library's own logarithm and sine / cosine (mppi_prelude.cuh), checked on
the CPU: the polynomial constants are read from the device source and
evaluated the way the device does (float32, fused multiply-adds emulated
exactly through float64 products; csrc/device/derive_poly.py), against
float64 log / sin / cos, to the error bounds the source states.  The GPU tests
(test_gpu_parity.py) check the compiled functions themselves."""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np

DEVICE = Path(__file__).resolve().parents[1] / "mppi_metal_b200" / "csrc" / "device"
sys.path.insert(0, str(DEVICE))
import derive_poly as dp  # noqa: E402

PRELUDE = (DEVICE / "mppi_prelude.cuh").read_text()
F = np.float32


def _body(name: str) -> str:
    start = PRELUDE.index(f"__device__ __forceinline__ {name}")
    return PRELUDE[start:PRELUDE.index("\n}\n", start)]


def _hexfloats(text: str) -> list:
    return [float.fromhex(h) for h in re.findall(r"-?0x1(?:\.[0-9a-f]+)?p[+-]?\d+", text)]


def test_log_constants_and_error():
    body = _body("float mppi_log(float x)")
    vals = _hexfloats(body)
    # Horner from the highest coefficient (c7, c6, ..., c0), then ln 2 hi / lo
    c = [F(v) for v in vals[:8]][::-1]
    ln2_hi, ln2_lo = F(vals[8]), F(vals[9])
    assert float(ln2_hi) == float(dp.LN2_HI) and float(ln2_lo) == float(dp.LN2_LO)
    assert "0x3f2aaaab" in body
    rel, _ = dp.check_log(c)
    assert rel < 1.0e-7


def test_quarter_turn_constants_and_error():
    body = _body("void mppi_sincos_quarter(float v, float* so, float* co)")
    h = [F(x) for x in _hexfloats(body)]
    # appearance: 0x1.8p23 (twice), s3, s2, s1, s0, c3, c2, c1, c0
    rnd = [x for x in h if float(x) == float.fromhex("0x1.8p23")]
    assert len(rnd) == 2
    coef = [x for x in h if float(x) != float.fromhex("0x1.8p23")]
    s3, s2, s1, s0, c3, c2, c1, c0 = coef
    es, ec = dp.check_quarter([s0, s1, s2, s3], [c0, c1, c2, c3])
    assert es < 1.0e-7 and ec < 1.0e-7


def test_radian_constants_and_error():
    body = _body("void mppi_sincosf(float x, float* so, float* co)")
    h = [F(x) for x in _hexfloats(body)]
    # appearance: 2/pi, 1.5 * 2^23 (twice), pi/2 in two parts, then the sine
    # polynomial S2, S1, S0 and the cosine polynomial C3, C2, C1 (C0 = -1/2)
    two_over_pi, split_hi, split_lo = h[0], h[3], h[4]
    assert float(two_over_pi) == float(F(2.0 / np.pi))
    assert float(split_hi) == float(F(np.pi / 2))
    assert float(split_lo) == float(F(np.pi / 2 - np.float64(split_hi)))
    s2, s1, s0, c3, c2, c1 = h[5], h[6], h[7], h[8], h[9], h[10]
    assert "-0.5f" in body
    es, ec = dp.check_radians([s0, s1, s2], [F(-0.5), c1, c2, c3])
    assert es < 1.0e-7 and ec < 1.0e-7
