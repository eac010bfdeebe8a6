import json
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / 'golden'
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line('markers',
                            'gpu: needs a CUDA device (B200 / sm_100a)')
    config.addinivalue_line('markers', 'slow: long-running test')


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason='no CUDA device')
    for item in items:
        if 'gpu' in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope='session')
def golden_kernels():
    with np.load(GOLDEN / 'fd_kernels.npz') as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope='session')
def golden_stencils():
    return json.loads((GOLDEN / 'stencils.json').read_text())


def seeded(seed, shape, cplx):
    """Inputs of tests/golden/make_golden.py (regenerated from the seed)."""
    rng = np.random.default_rng(seed)
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return a


def bloch_phases(pbc, k_c=(0.1, 0.25, -0.3)):
    sd = np.zeros((3, 2))
    p = np.asarray(pbc, bool)
    sd[p, 0] = 1
    sd[p, 1] = -1
    return np.exp(2j * np.pi * sd * np.asarray(k_c)[:, None])


def relerr(a, b):
    """Norm-wise relative error max|a - b| / max|b| (the parity measure)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale
