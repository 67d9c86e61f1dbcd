"""Test configuration: paths, the `gpu` marker, the checker build.

CPU tests (-m "not gpu") check the oracle against the reference's golden
vectors, the host logic and the C ABI of the library without calling any
kernel. GPU tests (-m gpu) are the parity tests proper: they call the CUDA
library through its C ABI and compare with the oracle.
"""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle", ROOT / "gpu-assembly_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    if not (ROOT / "oracle" / "_build" / "liboracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "oracle"], check=True)


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def ctx(torch_cuda):
    import rbf_b200
    c = rbf_b200.Context(0)
    yield c
    torch_cuda.cuda.synchronize()
    c.close()
