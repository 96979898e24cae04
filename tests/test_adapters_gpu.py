"""The C++ drop-ins (GpuBVHAccelerator, GpuPathIntegrator) used through the reference's own
Accelerator / Integrator interfaces, by the C++ programs in tests/cpp (built against the
reference headers by ray-based-rendering_b200/adapters/Makefile)."""
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BIN = Path(__file__).resolve().parent / "cpp" / "_bin"


@pytest.mark.parametrize("name", ["test_gpu_accelerator", "test_gpu_integrator", "test_gpu_accel_integrators"])
def test_cpp_adapter(name):
    exe = BIN / name
    if not exe.exists():
        pytest.skip(f"{exe} not built (needs the reference headers at build time)")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
