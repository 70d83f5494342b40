"""Test configuration: the `gpu` marker and shared fixtures.

`-m "not gpu"` runs the oracle, host-logic and ABI checks on any machine; `-m gpu` runs the
parity tests of the CUDA library against the oracle on a B200.
"""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libMKF.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import RefOracle

    if not RefOracle.available():
        pytest.skip("reference C library (oracle/_ref) not built on this machine")
    return RefOracle()


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(GOLDEN, "ref_cases.npz"))


@pytest.fixture(scope="session")
def mkf():
    import mkf_b200

    mkf_b200.lib()
    return mkf_b200


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    return torch.device("cuda:0")
