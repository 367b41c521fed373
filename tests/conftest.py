import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and libdrwc.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def ctx():
    """Device context on cuda:0 through the C ABI (GPU tests only)."""
    from deeprwcap_b200 import engine
    c = engine.default_context(0)
    yield c


def golden(N):
    import numpy as np
    return np.load(GOLDEN / f"ggft_N{N}.npz")
