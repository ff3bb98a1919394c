"""Shared fixtures: library bindings, the oracle, and small seeded scenes."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "insar-on-sentinel-1-tops-data_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def T():
    import topsb200
    return topsb200


@pytest.fixture(scope="session")
def O():
    import oracle
    return oracle


SMALL = dict(n_bursts=2, lines_per_burst=300, samples_per_burst=512, overlap_lines=30,
             dem_lines=192, dem_pixels=192, seed=11)


@pytest.fixture(scope="session")
def scene_small(T):
    return T.Scene(**SMALL)


@pytest.fixture(scope="session")
def scene_esd(T):
    """Three bursts with an injected azimuth misregistration (ESD known answer)."""
    return T.Scene(n_bursts=3, lines_per_burst=400, samples_per_burst=768, overlap_lines=40,
                   dem_lines=256, dem_pixels=256, seed=5, az_shift_true=0.05)


def rel_rms(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / max(np.sum(np.abs(b) ** 2), 1e-300)))


def c64(x):
    """complex128 [L][W] -> interleaved float32 [L][W][2]."""
    return np.ascontiguousarray(np.asarray(x, np.complex64)).view(np.float32).reshape(
        x.shape[0], x.shape[1], 2)
