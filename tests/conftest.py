import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_LIB = os.path.join(ROOT, "oracle", "_ref", "liboracle.so")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtioga_ref.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libtioga_b200.so")


@pytest.fixture(scope="session")
def oracle_lib():
    if not os.path.exists(ORACLE_LIB):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)
    return ORACLE_LIB
