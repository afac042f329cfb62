import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA engine")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    # The oracle restatement is test infrastructure; build it if absent.
    lib = os.path.join(ROOT, "oracle", "_build", "libhy_oracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "lib"], check=True)
    yield
