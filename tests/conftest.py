import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(os.path.join(GOLDEN, "oracle_cases.npz")))


@pytest.fixture(scope="session")
def known_answers():
    import json
    with open(os.path.join(GOLDEN, "reference_known_answers.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ctx():
    import torch
    import arma_b200 as A
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    torch.cuda.init()
    c = A.Context(0)
    yield c
    c.close()
