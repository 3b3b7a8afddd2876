"""Shared test setup: import path, the `gpu` marker, library fixtures."""

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "lcs.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _build(dirname, target):
    path = os.path.join(ROOT, dirname, target)
    if not os.path.exists(path):
        subprocess.run(["make", "-C", os.path.join(ROOT, dirname)], check=True, capture_output=True)
    return path


@pytest.fixture(scope="session")
def oracle_lib_path():
    return _build("oracle", "liblcs_oracle.so")


@pytest.fixture(scope="session")
def cuda_lib_path():
    return _build("lcs.jl_b200", "liblcs_b200.so")


def gpu_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
