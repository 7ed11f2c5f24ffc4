import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "cans-fizzy_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

# the reference checkout (present only in the build container); override
# with CANSFZ_REFERENCE_DIR
REFERENCE = os.environ.get("CANSFZ_REFERENCE_DIR", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test (several seconds)")


@pytest.fixture(scope="session")
def reference_dir():
    """The reference checkout, present only in the build container."""
    if not os.path.isdir(os.path.join(REFERENCE, "tests")):
        pytest.skip("reference checkout not present on this machine")
    return REFERENCE
