"""Test configuration: the `gpu` marker, and build-on-demand of the CPU
checkers (oracle/) and of libcc_b200.so."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def _built():
    from core_collapse_b200 import _lib as L
    if not L.LIB_PATH.exists():
        from core_collapse_b200.build import build
        build()
    import oracle_lib
    if not (oracle_lib.ORACLE_DIR / "liboracle.so").exists():
        oracle_lib.build_oracle()
    yield
