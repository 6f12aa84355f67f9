import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "chaste_kats.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libchastegpu.so")


@pytest.fixture(scope="session")
def kats():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_dir():
    import pathlib

    return pathlib.Path(ROOT) / "tests" / "golden"


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def native():
    """libchastegpu.so, built in-tree."""
    from chaste_b200 import _native
    from chaste_b200.build import build_native

    build_native()
    return _native
