"""Shared pytest setup: import paths, the ``gpu`` marker and fixture loaders."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for path in (ROOT, os.path.join(ROOT, "bempp-cl_b200")):
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def probe_vectors(rows, cols, seed=1234):
    """Same seeded probes as tests/golden/make_golden.py."""
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((cols, 2)) + 1j * rng.standard_normal((cols, 2))
    w = rng.standard_normal((rows, 2)) + 1j * rng.standard_normal((rows, 2))
    ii = rng.integers(0, rows, 48)
    jj = rng.integers(0, cols, 48)
    return u, w, ii, jj


def rel_fro(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="session")
def sphere_msh_grid():
    from bempp_cuda.grid import Grid

    d = load_golden("sphere_msh.npz")
    return Grid(d["vertices"], d["elements"], d["tags"])


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as orc

    orc.lib()
    return orc
