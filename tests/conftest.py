import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C-ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle.native import ORACLE_PATH, Oracle, build

    if not ORACLE_PATH.exists():
        build(reference=False)
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.native import REFERENCE_PATH, Reference, build

    if not REFERENCE_PATH.exists():
        if not Path("/root/reference/cpp").exists():
            pytest.skip("the reference library was not built and its sources are absent")
        build(reference=True)
    return Reference()


@pytest.fixture(scope="session")
def backend():
    from microsimulator_b200.backend import B200Backend

    b = B200Backend(int(os.environ.get("MSB_DEVICE", "0")))
    yield b
    b.close()


def load_golden(name):
    return np.load(GOLDEN / f"{name}.npz")


@pytest.fixture(scope="session")
def golden():
    return load_golden
