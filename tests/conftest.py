"""Test configuration: the `gpu` marker and import paths.

CPU tests (``-m "not gpu"``) check the oracle against the golden fixtures, the
host logic, and that libpfc_b200.so loads and exports every declared symbol.
GPU tests (``-m gpu``) are the parity tests proper: they call the CUDA engine
through its C ABI and compare with the oracle and the fixtures.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("", "oracle", "pfc-exp-gui_b200", "tests"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA engine")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.lib()
    return oracle
