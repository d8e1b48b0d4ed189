import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA path)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def ctx():
    from sabertooth_b200 import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(params=["host", "device"])
def planner(request, monkeypatch):
    """Runs a batched-scoring test once with the host planner and once with the
    device planner (every batch size planned on the GPU)."""
    if request.param == "host":
        monkeypatch.setenv("ST_DEVICE_PLAN", "0")
    else:
        monkeypatch.setenv("ST_DEVICE_PLAN", "1")
        monkeypatch.setenv("ST_DEVICE_PLAN_MIN", "1")
    return request.param
