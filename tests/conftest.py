"""Shared fixtures.  Tests marked `gpu` need a CUDA device (a B200); everything else runs on
the CPU: the oracle against the reference's golden vectors, the host logic, and the C ABI
exports of libmathpub.so."""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_vectors():
    return load_golden("ref_vectors.json")


@pytest.fixture(scope="session")
def verify_py():
    return load_golden("verify_py.json")


@pytest.fixture(scope="session")
def configs():
    return load_golden("configs.json")


@pytest.fixture(scope="session")
def engine():
    import mathpub_b200 as mp
    mp.build_if_needed = None
    e = mp.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.o()
    return oracle
