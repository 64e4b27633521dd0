import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA (sm_100a) device")
    config.addinivalue_line("markers", "slow: minutes of CPU; runs only with WIG_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("WIG_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow oracle pin; set WIG_SLOW=1")
    for it in items:
        if "slow" in it.keywords:
            it.add_marker(skip)
