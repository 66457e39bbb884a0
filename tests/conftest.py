import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (run on the B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import build as oracle_build
    from oracle.bindings import Oracle
    oracle_build.build_oracle()
    return Oracle()


@pytest.fixture(scope="session")
def golden_lbvh():
    import numpy as np
    data = np.load(os.path.join(ROOT, "tests", "golden", "lbvh_reference.npz"))
    cases = {}
    for key in data.files:
        name, field = key.split("/", 1)
        cases.setdefault(name, {})[field] = data[key]
    return cases


@pytest.fixture(scope="session")
def ctx():
    import lux_b200
    c = lux_b200.Context(0)
    yield c
    c.close()
