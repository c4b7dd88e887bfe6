import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ref_values():
    return json.loads((GOLDEN / "ref_values.json").read_text())


@pytest.fixture(scope="session")
def ref_lg1d():
    return dict(np.load(GOLDEN / "ref_lg1d.npz"))


# The 2-D LG model of the benchmark configurations:
# A = rot(0.2), Q = [[1,1e-4],[1e-4,1]]/100, R = [[1,.1],[.1,1]]/10, C = I, X0 = 0.
LG2_Q = np.array([[1.0, 1e-4], [1e-4, 1.0]]) / 100
LG2_R = np.array([[1.0, 0.1], [0.1, 1.0]]) / 10


@pytest.fixture
def lg2d():
    """A fresh model per test: methods record results on the object, so a
    shared one would carry one test's history into the next."""
    import pypomp_b200 as pp

    return pp.LG(T=50, Q=LG2_Q, R=LG2_R, key=0)
