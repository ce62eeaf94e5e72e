"""Shared test setup: import paths, markers, and cached problem builders."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "hacapk-magma_b200"))
sys.path.insert(0, ROOT)

REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100)")


@pytest.fixture(scope="session")
def build_libs():
    """The two package libraries and the oracle are built once per session."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "hacapk-magma_b200")], check=True)
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return True


_cache = {}


def sphere(level, leaf_size=32, eta=2.0, aca_eps=1e-5, kernel=None):
    from hacapk_b200 import abi, hmatrix
    key = (level, leaf_size, eta, aca_eps, kernel)
    if key not in _cache:
        k = abi.KERNEL_LAPLACE if kernel is None else kernel
        _cache[key] = hmatrix.HostHMatrix(hmatrix.icosphere(level), leaf_size=leaf_size, eta=eta,
                                          aca_eps=aca_eps, kernel=k)
    return _cache[key]


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
