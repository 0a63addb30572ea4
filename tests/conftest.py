import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "ref_runs.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def libpath():
    """The in-tree library; built here when missing (nvcc cross-compiles without a GPU)."""
    from brisk_b200 import build
    lib = os.path.join(ROOT, "brisk_b200", "libbrisk.so")
    if not os.path.exists(lib):
        build.build()
    return lib


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    return torch.device("cuda:0")
