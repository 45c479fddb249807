"""Shared test set-up: the `gpu` marker, the repo root on sys.path, and an
incremental build of the library and the parity checkers."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a); run with -m gpu")
    for d in ("ozablas_b200/csrc", "oracle", "baseline"):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, d)], check=True,
                       stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def executor():
    import ozablas_b200 as oz
    return oz.CudaExecutor(0)
