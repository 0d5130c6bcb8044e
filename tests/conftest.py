"""Shared pytest configuration.

``-m gpu`` tests need a CUDA device and call the product through its C ABI
(via the Python drop-in layer); everything else runs on the CPU: the oracle
against the reference's golden vectors, host-side logic, and the C ABI
library's symbol table.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running parity case")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


from integer_delauney_b200.workloads import clustered as clustered_seeds  # noqa: E402,F401
from integer_delauney_b200.workloads import uniform as _uniform  # noqa: E402


def random_seeds(W, H, n, seed, margin=0):
    """n distinct integer seeds, uniform on [margin, W-margin) x [margin, H-margin)."""
    return _uniform(W, H, n, seed, margin)


@pytest.fixture(scope="session")
def golden_dir():
    return os.path.join(ROOT, "tests", "golden")
