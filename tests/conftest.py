import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built vlgpu extension")


@pytest.fixture(scope="session")
def mesh():
    from vlasiator_b200.mesh import VelocityMesh
    return VelocityMesh()


@pytest.fixture(scope="session")
def orc_sp():
    from oracle.oracle import Restatement
    return Restatement("sp")


@pytest.fixture(scope="session")
def orc_dp():
    from oracle.oracle import Restatement
    return Restatement("dp")
