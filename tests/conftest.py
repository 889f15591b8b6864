import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libaero2d_b200.so")
    config.addinivalue_line("markers", "slow: long CPU oracle runs (minutes)")


@pytest.fixture(scope="session")
def ref_grids():
    return dict(np.load(GOLDEN / "ref_grids.npz"))


@pytest.fixture(scope="session")
def known_answers():
    import json
    return json.load(open(GOLDEN / "ref_known_answers.json"))


@pytest.fixture(scope="session")
def converged_0012():
    return dict(np.load(GOLDEN / "naca0012_128x48_r40_converged.npz"))


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from aero2d_b200 import _lib
    _lib.load()          # a GPU machine without the built library must fail, not skip
    return torch.device("cuda", 0)
