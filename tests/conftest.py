"""Shared fixtures: the B200 library (libssol_b200.so) and the CPU oracle
(oracle/_build/liboracle_ssol.so), both driven through the same ctypes
binding of the ssol C API."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "solstice-solver_b200")
sys.path.insert(0, PKG)

import pyssol  # noqa: E402

ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle_ssol.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                       stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    return ORACLE_LIB


def _ensure_product():
    if not os.path.exists(pyssol.PRODUCT_LIB):
        sys.path.insert(0, PKG)
        import build  # noqa: F401
        build.build()
    return pyssol.PRODUCT_LIB


@pytest.fixture(scope="session")
def oracle():
    return pyssol.Lib(_ensure_oracle())


@pytest.fixture(scope="session")
def product():
    return pyssol.load_product(_ensure_product())


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
