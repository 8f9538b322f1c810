"""Shared test set-up: import paths, the `gpu` marker, fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "sph-code-simulation_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) device")


@pytest.fixture(scope="session")
def G():
    import sphgpu
    sphgpu.lib()
    return sphgpu


@pytest.fixture(scope="session")
def O():
    import oracle
    if not os.path.exists(oracle.ORACLE_LIB):
        oracle.build(reference=False)
    return oracle


@pytest.fixture(scope="session")
def gpu(G):
    if not G.device_ok():
        pytest.fail("no usable sm_100 device for a gpu-marked test")
    return G


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def params_from_bytes(G, raw):
    """Parameters stored as raw struct bytes; fields appended to the struct
    after the fixture was written keep their defaults.  tree_root_origin
    took over 4 bytes of padding, so fixtures written before it read 0 there
    (the particles' own root box); their particles span the origin or the box
    is periodic, where both root boxes are the same."""
    import ctypes
    p = G.default_params()
    b = bytes(raw.tobytes())
    ctypes.memmove(ctypes.byref(p), b, min(len(b), ctypes.sizeof(p)))
    return p


def rel_err(a, b, floor=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.maximum(np.abs(b), floor if floor is not None else 1e-300)
    return np.abs(a - b) / scale
