import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_bin():
    """The CPU restatement CLI, built from oracle/ on demand (gcc only)."""
    path = os.path.join(ROOT, "oracle", "build", "poa_oracle")
    lib = os.path.join(ROOT, "oracle", "build", "libpoa_oracle.so")
    if not (os.path.exists(path) and os.path.exists(lib)):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "restatement"], check=True)
    return path
