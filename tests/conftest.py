import importlib
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
PKG_NAME = "tinysolverdx-batched-small-matrix-cholesky-lu-with-numerical_b200"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_pkg(sub=None):
    return importlib.import_module(PKG_NAME + ("." + sub if sub else ""))


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle, PORT_LIB, build
    if not PORT_LIB.exists():
        build(reference=False)
    return Oracle("port")


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(ROOT / "tests" / "golden" / "golden.npz")
