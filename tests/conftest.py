import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs through libraishin_gpu.so")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    if not has_gpu():
        pytest.skip("no CUDA device")
    from raishinsource_b200 import Context
    ctx = Context(0)
    yield ctx
    ctx.close()


def field_err(a: np.ndarray, b: np.ndarray, region=None) -> np.ndarray:
    """Per-variable max |a-b| / max |b| over a region (slices over (k, j, i))."""
    if region is not None:
        a, b = a[region], b[region]
    a = a.reshape(-1, a.shape[-1])
    b = b.reshape(-1, b.shape[-1])
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(a - b).max(axis=0) / scale
