import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "gdistger-re_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import dgoracle
    dgoracle.build()
    return dgoracle


@pytest.fixture(scope="session")
def distger_lib():
    import distger
    if not os.path.exists(distger._lib.LIB_PATH):
        distger.build()
    return distger
