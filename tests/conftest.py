import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, 'tests', 'golden', 'fd_golden.npz')


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA GPU (runs the sm_100a library)')


@pytest.fixture(scope='session')
def golden():
    return np.load(GOLDEN)


def rel_err(a, b):
    """max |a - b| / max |b| (the parity measure for stencils and transfers)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = np.abs(b).max()
    return float(np.abs(a - b).max() / (scale if scale > 0 else 1.0))


@pytest.fixture(scope='session')
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail('GPU test run without a CUDA device')
    return torch.device('cuda:0')
