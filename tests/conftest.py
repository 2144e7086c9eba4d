"""Shared pytest setup: markers, paths and fixtures."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "dmg-md_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def potential(name):
    return os.path.join(GOLDEN, "potentials", name)


@pytest.fixture(scope="session")
def goldens():
    with open(os.path.join(GOLDEN, "baseline_goldens.json")) as f:
        return json.load(f)
