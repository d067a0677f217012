"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device (run with ``-m gpu``); everything else
runs on the CPU (``-m "not gpu"``).  The oracle under oracle/ is the checker
for both and is built on first use.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as o

    if not os.path.exists(o.ORACLE_SO):
        o.build_oracle()
    return o


@pytest.fixture(scope="session")
def sbf():
    import cusbf_b200

    return cusbf_b200


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test selected but no CUDA device is visible")
    torch.cuda.init()
    return torch


def random_dna(rng, n, alphabet=b"ACGT"):
    a = np.frombuffer(alphabet, dtype=np.uint8)
    return a[rng.integers(0, len(a), size=n, dtype=np.int64)]
