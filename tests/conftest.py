"""Shared test configuration.

Tests marked ``gpu`` need a CUDA device (a B200); everything else runs on the
CPU: the oracle against the golden fixtures and known answers, the host logic,
and the C ABI's symbol table.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the oracle and the GPU library in-tree if they are missing."""
    for sub, lib in [("oracle", "liboracle.so"), ("pmpic_b200", "libpmpic_gpu.so"),
                     ("pmpic_b200", "pmpic_monc")]:
        if not os.path.exists(os.path.join(ROOT, sub, lib)):
            subprocess.run(["make", "-s", "-C", os.path.join(ROOT, sub)], check=True)
    yield


GOLDEN = os.path.join(ROOT, "tests", "golden")
