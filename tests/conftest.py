import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "multigrid-poisson_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session")
def mgp_mod():
    import mgp

    return mgp


@pytest.fixture(scope="session")
def gpu_ready(mgp_mod):
    n = mgp_mod.device_count()
    if n < 1:
        pytest.fail("no CUDA device visible to the engine (GPU tests must run on a GPU box)")
    return n
