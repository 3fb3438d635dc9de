"""Test configuration: import paths, the ``gpu`` marker, checker builds."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "p2c-ccd_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    if not oracle.ORACLE_SO.exists():
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a CUDA device is required for gpu-marked tests")
    return torch.device("cuda:0")
