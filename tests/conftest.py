"""Shared pytest configuration.

Tests marked ``gpu`` need a B200 and call the engine through the C ABI; every other test runs on
a CPU-only machine.  The oracle (oracle/) is the checker in both kinds of test.
"""

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


@pytest.fixture(scope="session")
def gpu_device():
    import fresnel_b200
    return fresnel_b200.Device(mode="gpu")


@pytest.fixture(scope="session")
def oracle_device():
    from oracle import cpu_module
    return cpu_module.make_device("restated")
