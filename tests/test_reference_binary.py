"""The reference's own test program (tests/mppi_driver_tests.cpp of
MarshallVielmetti/mppi_metal), compiled unchanged against this project's
headers and linked to libmppi_b200.so (oracle/Makefile target `ref_suite`,
built where the reference tree exists; the binary travels with the tree).
TEST_USER_METALLIB_PATH points at the CUDA form of the reference's test
plugin.  Every one of its checks must pass on the B200 backend."""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

import pytest

BIN = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "mppi_driver_tests"


@pytest.mark.gpu
@pytest.mark.skipif(not BIN.exists(), reason="reference test program not built (make -C oracle ref_suite)")
def test_reference_test_program_passes_unchanged():
    r = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    out = r.stdout + r.stderr
    m = re.search(r"(\d+) passed, (\d+) failed", out)
    assert m, out[-2000:]
    passed, failed = int(m.group(1)), int(m.group(2))
    assert failed == 0, "\n".join(l for l in out.splitlines() if "[FAIL]" in l)
    assert passed >= 70
    assert r.returncode == 0
