"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device and run the product library; all
others run on the CPU (oracle, host set-up, C-ABI exports)."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and runs libsemba_gpu kernels")


def pytest_sessionstart(session):
    # build the oracle (and, where nvcc exists, the CUDA libraries) once
    import subprocess
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)


@pytest.fixture(scope="session")
def casedir(tmp_path_factory):
    return tmp_path_factory.mktemp("cases")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
