"""Shared test setup: import paths, the ``gpu`` marker, fixtures.

``-m "not gpu"`` tests run anywhere (oracle vs golden vectors, host logic,
library exports); ``-m gpu`` tests need a CUDA GPU and call the product
through its C ABI.
"""
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "simple-cpsd_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))
GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def restatement():
    import oracle
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "restatement"], check=True)
    return oracle.Restatement()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return np.load(os.path.join(GOLDEN, "ref_%s.npz" % name))
    return load
