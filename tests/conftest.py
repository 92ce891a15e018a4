import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, HERE)
sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle():
    # make rebuilds the oracle only when a source is newer than it
    subprocess.check_call(["make", "-s", "-C", os.path.join(REPO, "oracle")])
    return os.path.join(REPO, "oracle", "liboracle.so")


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle_ctypes import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def oracle_gxm():
    """The oracle's parity build (gx_math.h's elementary functions)."""
    _ensure_oracle()
    from oracle_ctypes import ORACLE_GXM_SO, Oracle
    return Oracle(ORACLE_GXM_SO)


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    d = os.path.join(HERE, "golden")
    return {k: np.load(os.path.join(d, k + ".npz")) for k in
            ("mrg", "tables", "models_quirk", "xs", "processes", "helix")}
