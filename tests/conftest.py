import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU run; enabled with ASTR_SLOW=1")


def pytest_collection_modifyitems(config, items):
    if os.environ.get("ASTR_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="slow; set ASTR_SLOW=1")
    for it in items:
        if "slow" in it.keywords and "gpu" not in it.keywords:
            it.add_marker(skip)
