import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def small_cfg(**over):
    """A small cone-beam geometry: 32x32x24 volume, 64x48 detector, 12 views."""
    from recon_b200.configs import CPU_SMALL, scaled

    base = dict(Xdim=32, Ydim=32, Zdim=24, XVoxSize=1.0, YVoxSize=1.0, ZVoxSize=1.0, AxPixels=64, TAxPixels=48,
                AxPixDim=1.5, TAxPixDim=1.5, NumProj=12)
    base.update(over)
    return scaled(CPU_SMALL, **base)


@pytest.fixture
def small():
    return small_cfg()


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
