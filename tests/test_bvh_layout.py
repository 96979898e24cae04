"""The wide-BVH builder on the CPU: tests/cpp/test_bvh_layout.cpp, compiled here against
ray-based-rendering_b200/csrc/bvh_build.cpp, checks the node layout the traversal kernels rely
on and replays their traversal order on the host against brute force (triangle soups: uniform,
coplanar, duplicated, mixed sizes; axis-aligned rays). No GPU is involved."""
import shutil
import subprocess
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
CSRC = REPO / "ray-based-rendering_b200" / "csrc"
SRC = REPO / "tests" / "cpp" / "test_bvh_layout.cpp"
BIN = REPO / "tests" / "cpp" / "_bin" / "test_bvh_layout"


@pytest.fixture(scope="module")
def exe():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    BIN.parent.mkdir(exist_ok=True)
    r = subprocess.run([cxx, "-O2", "-std=c++17", f"-I{CSRC}", str(SRC), str(CSRC / "bvh_build.cpp"), "-o", str(BIN),
                        "-lpthread"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return BIN


def test_wide_bvh_layout_and_traversal_replay(exe):
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 8 and all(l.endswith(" 0 mismatches") for l in lines), r.stdout
    # every case (the 1- and 7-triangle trees included) is exercised by many hitting rays:
    # half of the rays aim at a random triangle's centroid
    hits = [int(l.split(" rays hit")[0].split(", ")[-1].split(" of ")[0]) for l in lines]
    assert min(hits) >= 600, r.stdout
