import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(autouse=True, scope="module")
def _release_device_caches():
    """Each test module leaves no cached plans behind: the nside 4096 plans of one module would
    otherwise hold device memory that a later module's batched plan needs."""
    yield
    hb = sys.modules.get("hellblast_b200")
    if hb is not None:
        hb.clear_caches()


@pytest.fixture(scope="session")
def oracle():
    from oracle import sht_oracle
    return sht_oracle


GOLDEN = os.path.join(ROOT, "tests", "golden")
