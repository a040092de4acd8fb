"""Test configuration: the `gpu` marker and the in-tree builds."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200)")


@pytest.fixture(scope="session", autouse=True)
def native_builds():
    """Build the library and the oracle if their sources changed (no-op otherwise)."""
    from voxviz_b200 import build as vb
    from oracle import gv_oracle

    vb.build()
    gv_oracle.build()
    yield
