import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU check")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Oracle, build
    if not Oracle.available("port"):
        build()
    return Oracle("port")


@pytest.fixture(scope="session")
def golden_small():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "ref_small.npz"))


@pytest.fixture(scope="session")
def golden_plain():
    import numpy as np
    return dict(np.load(ROOT / "tests" / "golden" / "ref_plain_end_to_end.npz"))
