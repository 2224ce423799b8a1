import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
PKG = REPO / "walking-into-holes_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"
for p in (str(PKG), str(REPO / "oracle"), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def bunny1000(oracle_mod):
    return oracle_mod.load_ascii_ply(GOLDEN / "bunny-01000-faces.ply.gz")


@pytest.fixture(scope="session")
def eval_points(oracle_mod):
    return oracle_mod.read_points(GOLDEN / "compiled_bunny" / "evaluation-points.csv")


@pytest.fixture(scope="session")
def housing(oracle_mod):
    return oracle_mod.load_ascii_ply(GOLDEN / "stylized-finned-housing.ply.gz")


@pytest.fixture(scope="session")
def lib_built():
    import build
    build.build()
    return True
