import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "grid-calculus_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib
    return oracle_lib.oracle()


@pytest.fixture(scope="session")
def gc():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import gridcalc_b200
    return gridcalc_b200


@pytest.fixture(scope="session")
def dev():
    import torch
    return torch.device("cuda:0")
