import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")
    config.addinivalue_line("markers", "slow: long CPU replay, runs only with ECSG_SLOW=1")


def _gpu_count():
    try:
        import ecsg_b200
        return ecsg_b200.lib().ecsg_device_count()
    except Exception:
        return 0


def pytest_collection_modifyitems(config, items):
    slow_ok = os.environ.get("ECSG_SLOW") == "1"
    have_gpu = None
    for it in items:
        if "slow" in it.keywords and not slow_ok:
            it.add_marker(pytest.mark.skip(reason="set ECSG_SLOW=1 for the full-length CPU replays"))
        if "gpu" in it.keywords:
            if have_gpu is None:
                have_gpu = _gpu_count() > 0
            if not have_gpu:
                it.add_marker(pytest.mark.skip(reason="no CUDA device"))


def ref_available(bits=64):
    from oracle import ref
    return ref.available(bits)
