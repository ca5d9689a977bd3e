import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import build, oracle
    build.build_oracle()
    return oracle


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built if missing; GPU tests fail (not skip) when it cannot load."""
    from physica_b200 import build, pbf
    build.build()
    return pbf
