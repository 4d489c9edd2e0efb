import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def ref_meshes():
    """libsupermesh's own test meshes (tests/golden/make_fixtures.py)."""
    data = np.load(ROOT / "tests" / "golden" / "ref_meshes.npz")

    def get(name):
        return data[f"{name}/positions"], data[f"{name}/enlist"]

    return get


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def gpu_ctx():
    import libsupermesh_b200 as lsm

    ctx = lsm.Context(0)
    yield ctx
    ctx.close()
