"""pytest configuration: the ``gpu`` marker and shared fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libspectgpu.so")


@pytest.fixture(scope="session")
def S():
    """The package (spectrecon.jl_b200 imported as spectrecon_b200)."""
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (checker)."""
    from oracle import oracle

    return oracle


def sym_psfs(rng, px, pz, ny, nview):
    """Random point-symmetric PSFs normalised per plane (test/adjoint-project.jl:20-24)."""
    p = rng.random((px, pz, ny, nview))
    p = p + p[::-1, ::-1]
    p = p / p.sum(axis=(0, 1), keepdims=True)
    return np.asfortranarray(p, np.float32)


def relerr(a, b):
    """max |a-b| / max |b| (the error definition used for parity)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
