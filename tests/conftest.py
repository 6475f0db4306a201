import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) CUDA device")
    config.addinivalue_line("markers", "ref: needs the reference adapter oracle/_ref/libclothref.so")


@pytest.fixture(scope="session")
def ctx_factory():
    from clothsimulator_b200 import native

    made = []

    def make(sheets):
        c = native.Context(0)
        c.load(sheets)
        made.append(c)
        return c

    yield make
    for c in made:
        c.close()
