import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

REFERENCE = os.environ.get("SNELLY_REFERENCE", "")  # a checkout of the reference, if any


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (runs the CUDA path through libsnelly)")
    config.addinivalue_line("markers", "reference: needs the reference checkout (builds its shader for the CPU)")


def pytest_collection_modifyitems(config, items):
    if not (REFERENCE and os.path.isdir(os.path.join(REFERENCE, "shaders"))):
        skip = pytest.mark.skip(reason="no reference checkout ($SNELLY_REFERENCE unset or not a checkout)")
        for it in items:
            if "reference" in it.keywords:
                it.add_marker(skip)


@pytest.fixture(scope="session")
def gpu_ctx():
    from snelly_b200 import api
    return api.Context(0)
