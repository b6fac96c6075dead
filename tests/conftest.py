"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs everything that needs no GPU (the oracle against the reference's
golden vectors, the residual judges, the C-ABI loading/exports and host-only argument
checks).  `-m gpu` runs the parity tests proper through the C ABI on a B200.
"""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "ops-solver_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("this test needs a CUDA device")
    torch.cuda.init()
    return torch.device("cuda:0")


@pytest.fixture()
def handle(cuda):
    import aclsolver

    h = aclsolver.Handle()
    yield h
    h.close()
