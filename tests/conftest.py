"""Shared pytest configuration.

Markers: ``gpu`` tests need a CUDA device (a B200) and call libsfac.so
through its C ABI; everything else runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libsfac.so")


def _cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def libsfac_path():
    """Path of libsfac.so, building it (nvcc, sm_100a) if it is missing."""
    from ewaldcorrel_b200 import build

    if not os.path.exists(build.LIB):
        build.build()
    return build.LIB


@pytest.fixture(scope="session")
def oracle_built():
    """Builds the CPU oracle (liborc.so) if it is missing."""
    import subprocess

    lib = os.path.join(ROOT, "oracle", "liborc.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "all"], check=True,
                       capture_output=True)
    return lib
