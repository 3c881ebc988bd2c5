"""Shared fixtures.

* ``oracle`` — the CPU restatement of the reference (oracle/), bound through
  the same Python API as the CUDA library; used only as the checker.
* ``gpu`` — the CUDA library; tests that need it carry ``@pytest.mark.gpu``.
"""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def build_oracle() -> Path:
    so = ROOT / "oracle" / "_build" / "liboracle.so"
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return so


@pytest.fixture(scope="session")
def oracle_lib():
    from scrs_b200.api import Library

    return Library(build_oracle(), prefix="oracle_", device=False)


@pytest.fixture(scope="session")
def oracle(oracle_lib):
    from scrs_b200.api import Api

    return Api(oracle_lib)


@pytest.fixture(scope="session")
def oracle_raw(oracle_lib):
    """The oracle's ctypes handle, for oracle-only probe entry points."""
    return oracle_lib.lib


@pytest.fixture(scope="session")
def gpu():
    import scrs_b200

    return scrs_b200.api_default()
