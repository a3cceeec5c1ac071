"""Test configuration: the `gpu` marker, import paths, and shared fixtures.

`-m "not gpu"` runs on any machine (oracle pins, host logic, library loading and exports);
`-m gpu` needs a B200 and calls the CUDA library through its C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "zk-gpu_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a library)")
    config.addinivalue_line("markers", "slow: large inputs (full benchmark sizes)")


@pytest.fixture(scope="session")
def gpu():
    from zk_gpu import Gpu
    return Gpu()
