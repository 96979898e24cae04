"""The path tracer's float sine and cosine (ray-based-rendering_b200/csrc/rbr_trig.h) on the
CPU: tests/cpp/test_trig.cpp compiles the same header for the host (explicit fused
multiply-adds, no contraction, so the host and device builds give the same bits) and measures
its error against double-precision sin/cos. The sampling routines pass angles in [-pi, 2 pi];
the bound of 1 ulp is checked on |x| <= 8. No GPU is involved."""
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
CSRC = REPO / "ray-based-rendering_b200" / "csrc"
SRC = REPO / "tests" / "cpp" / "test_trig.cpp"
BIN = REPO / "tests" / "cpp" / "_bin" / "test_trig"


@pytest.fixture(scope="module")
def exe():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    BIN.parent.mkdir(exist_ok=True)
    r = subprocess.run([cxx, "-O2", "-std=c++17", "-ffp-contract=off", f"-I{CSRC}", str(SRC), "-o", str(BIN)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return BIN


def test_sincos_within_one_ulp(exe):
    # every 5th float of [2^-12, 8] in both signs (about 52 M arguments; stride 1, all of them,
    # gives a largest error of 0.725 ulp for sin and 0.727 for cos)
    r = subprocess.run([str(exe), "5"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    n, max_s, at_s, max_c, at_c, cr = r.stdout.split()
    assert int(n) > 50_000_000
    assert float(max_s) < 0.75, f"sin: {max_s} ulp at {at_s}"
    assert float(max_c) < 0.75, f"cos: {max_c} ulp at {at_c}"
    # nearly always the correctly rounded float, as the double-precision library rounded once
    assert float(cr) > 0.99
