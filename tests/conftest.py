"""Shared fixtures.  GPU tests are marked `gpu` and run only on a B200 box
(`pytest -m gpu`); everything else runs on CPU (`pytest -m "not gpu"`)."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "nkr-zkp_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref (the reference built from source) is not built here")
    return oracle.Ref()


@pytest.fixture(scope="session")
def ctx():
    import nkr_b200
    c = nkr_b200.Context(0)
    yield c
    c.close()


@pytest.fixture
def rng():
    return np.random.default_rng(12345)
