import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "gr-athena_b200"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests", "golden"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the oracle library (seconds) and the CUDA library (cross-compiled
    for sm_100a; no GPU needed) when they are missing or stale."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    import build as cuda_build  # gr-athena_b200/build.py
    cuda_build.build()
    yield
