"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built CUDA library; the rest
run on the CPU (oracle pinning, host logic, C-ABI symbol checks, multi-rank
gloo tests).
"""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(REPO, "tests", "golden")
for _d in (os.path.join(REPO, "tests"), os.path.join(REPO, "oracle"), os.path.join(REPO, "hams-mrel_b200")):
    if _d not in sys.path:
        sys.path.insert(0, _d)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built hams_b200 CUDA library")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle, built on first use."""
    import oracle_lib

    return oracle_lib.load()


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


def build_oracle():
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle")], check=True)
