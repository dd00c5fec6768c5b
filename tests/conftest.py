import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "lbm-benchmark-kernels_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")
    config.addinivalue_line("markers", "big: full-size workload (runs in the -m gpu pass; minutes of host CPU)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, reference_available
    if not reference_available("verify"):
        pytest.skip("reference build oracle/_ref not present")
    r = Reference("verify")
    r.set_threads(min(4, os.cpu_count() or 1))
    return r
