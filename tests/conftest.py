"""Test configuration: markers, and the two libraries under comparison.

`product` is libmonolis_b200.so (the thing tested); `oracle` is the CPU
restatement of the reference (oracle/_build/libmonolis_oracle.so), used only
as the checker.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libmonolis_oracle.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    from monolis_b200 import api
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    if not os.path.exists(api.PRODUCT_SO):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "monolis_b200", "csrc")])


@pytest.fixture(scope="session")
def oracle():
    _ensure_built()
    from monolis_b200 import api
    lib = api.load_library(ORACLE_SO, oracle=True)
    lib.oracle_set_threads(1)  # serial sums: the reference's default build
    return lib


@pytest.fixture(scope="session")
def product():
    _ensure_built()
    from monolis_b200 import api
    return api.load_product()


@pytest.fixture(scope="session")
def gpu(product):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return product
