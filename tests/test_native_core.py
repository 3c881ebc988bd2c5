"""Builds tests/native/core_host_test.cu with nvcc as host code and runs it:
the bit-sliced multiply networks used by the sm_100a kernels must equal
scalar GF(256)/GF(65536) multiplication for every coefficient."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_bitsliced_core_matches_scalar_field(tmp_path):
    exe = tmp_path / "core_host_test"
    subprocess.run(["nvcc", "-O1", "-std=c++17", "-x", "cu", str(HERE / "native" / "core_host_test.cu"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASS" in r.stdout
