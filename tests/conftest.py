"""Test configuration: the `gpu` marker, the repository on sys.path, and the
checker fixtures (the oracle restatement and, when built, the reference)."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import REF_SO, Reference

    if not REF_SO.exists():
        pytest.skip("the reference driver oracle/_ref is not built (reference sources absent)")
    return Reference()


@pytest.fixture(scope="session")
def golden():
    from helpers import Golden

    return Golden()
