import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not oracle.LIB.exists():
        oracle.build(ref=False)
    return oracle


@pytest.fixture(scope="session")
def vrt():
    import voxelrt_b200
    return voxelrt_b200
