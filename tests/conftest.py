import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Selection tests check the built-in heuristic; the shipped predictor network
# and tuned table (loaded by the library on first use unless HML_PREDICTOR /
# HML_TUNED say otherwise) are exercised by their own tests, which load them
# explicitly or in a child process with the variable unset.
os.environ.setdefault("HML_PREDICTOR", "none")
os.environ.setdefault("HML_TUNED", "none")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
