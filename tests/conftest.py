"""pytest configuration: the ``gpu`` marker and shared fixtures.

Tests marked ``gpu`` need a B200 (sm_100a) and the in-tree CUDA library; all
other tests run on the CPU (oracle, host logic, C-ABI symbol checks).
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 GPU (sm_100a)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)
