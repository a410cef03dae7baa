import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libh3d.so")


def smooth_density(n, seed=0, vol=0.3):
    """Physical density rho^3 of the seeded trig-basis design, lexicographic float64."""
    from homo3d_b200.density import synthetic_density
    return synthetic_density(n, seed=seed, vol=vol).ravel() ** 3


def random_field(nv, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, size=(nv, 6, 3))


def to_lib_field(a):
    """oracle [nv, 6, 3] -> library [6, nv, 3] float32"""
    return np.ascontiguousarray(np.transpose(a, (1, 0, 2)), dtype=np.float32)


def from_lib_field(a):
    """library [6, nv, 3] -> oracle [nv, 6, 3] float64"""
    return np.ascontiguousarray(np.transpose(a, (1, 0, 2)), dtype=np.float64)


def half_ulp(x):
    """unit in the last place of FP16 at |x| (normal range), elementwise"""
    ax = np.maximum(np.abs(x), 6.1e-5)
    return 2.0 ** (np.floor(np.log2(ax)) - 10)


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for gpu tests")
    return torch
