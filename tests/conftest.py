import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
EXAMPLE_DIR = os.path.join(GOLDEN, "example")
ABX3_DIR = os.path.join(GOLDEN, "abx3")
# softplus/ReLU layers and non-integer zeta (tests/golden/make_prz_potential.py)
PRZ_DIR = os.path.join(GOLDEN, "prz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def pkg():
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def W(pkg):
    return pkg.workloads


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    return O


@pytest.fixture(scope="session")
def ex_model(orc):
    return orc.Model(EXAMPLE_DIR)


@pytest.fixture(scope="session")
def abx3_model(orc):
    return orc.Model(ABX3_DIR)


@pytest.fixture(scope="session")
def prz_model(orc):
    return orc.Model(PRZ_DIR)


@pytest.fixture(scope="session")
def c1(W):
    return W.config_c1(EXAMPLE_DIR)
