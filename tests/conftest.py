import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build (or reuse) the in-tree engine and oracle libraries."""
    from sensemap_b200 import build as engine_build
    from oracle import build as oracle_build
    engine_build.build()
    oracle_build.build()
