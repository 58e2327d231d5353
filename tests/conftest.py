import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")
    config.addinivalue_line("markers", "slow: longer CPU case")


@pytest.fixture(scope="session")
def oracle():
    from oracle import load_oracle
    return load_oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import load_reference, reference_available
    if not reference_available():
        pytest.skip("reference kernels not buildable here (no source tree, no prebuilt libcpsref.so)")
    return load_reference()
