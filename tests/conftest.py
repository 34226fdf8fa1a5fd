"""Shared fixtures of the test suite.

Markers: tests that need a CUDA device carry @pytest.mark.gpu; everything else runs on CPU.
The oracle (oracle/oracle.py over liboracle.so) is the checker; golden fixtures under
tests/golden/ were produced by the reference itself (tests/golden/make_golden.py).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def parse_sector(name):
    """(N, 2S, 2Lz) from a fixture name containing n<N>_2s<2S>_lz<2Lz>."""
    import re
    m = re.search(r"n(\d+)_2s(\d+)_lz(-?\d+)", name)
    return int(m.group(1)), int(m.group(2)), int(m.group(3))


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def dh():
    """The product package with its native library loaded (built if needed)."""
    import diagham_b200
    from diagham_b200 import _build
    _build.build()
    diagham_b200.load()
    return diagham_b200


@pytest.fixture(scope="session")
def gpu(dh):
    n = dh.device_count()
    if n < 1:
        try:
            import torch
            visible = torch.cuda.is_available()
        except Exception:
            visible = False
        if visible:
            pytest.fail("a CUDA device is visible but libdiagham_b200 sees none")
        pytest.skip("no CUDA device")
    return dh
