import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port
    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref
    if not Ref.available():
        pytest.skip("the reference core is not built here (oracle/_ref)")
    return Ref()


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN / "reference_outputs.npz"))


@pytest.fixture(scope="session")
def bessel_golden():
    return dict(np.load(GOLDEN / "bessel_reference.npz"))


@pytest.fixture(scope="session")
def lib():
    """The engine's C ABI on cuda:0 (GPU tests only)."""
    import spin_systems_b200 as ss
    return ss.load()


@pytest.fixture(scope="session")
def engine(lib):
    import spin_systems_b200 as ss
    eng = ss.Engine(0)
    yield eng
    eng.close()
