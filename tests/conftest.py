"""Shared test set-up: import paths, the gpu marker, built libraries."""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "3d-mfcfd_b200")
for p in (PKG, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _make(path):
    subprocess.run(["make", "-s", "-C", path], check=True, stdout=subprocess.DEVNULL)


@pytest.fixture(scope="session")
def oracle_lib():
    _make(os.path.join(REPO, "oracle"))
    from oracle import oracle
    return oracle


@pytest.fixture(scope="session")
def mfcfd_lib():
    lib_path = os.path.join(PKG, "mfcfd", "libmfcfd.so")
    if not os.path.exists(lib_path):
        _make(PKG)
    from mfcfd import _lib
    return _lib


@pytest.fixture(scope="session")
def small_cloud():
    from mfcfd import cloud
    return cloud.small_sphere()


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
