"""Shared fixtures. `-m gpu` tests need a CUDA device and the built librbr_b200.so; the rest
run on CPU (the oracle, the reference library built from source, host logic, the ABI)."""
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(REPO / "ray-based-rendering_b200"))
sys.path.insert(0, str(REPO / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and librbr_b200.so (runs on the B200 box)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def ctx():
    from rbr_b200 import Context

    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def restatement():
    from oracle import Restatement

    return Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, have_reference

    if not have_reference():
        pytest.skip("oracle/_ref/librbr_ref.so not built (needs the reference sources)")
    return Reference()
