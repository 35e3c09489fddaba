"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _build_library():
    lib = os.path.join(ROOT, "cvc_b200", "libcvcb200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", os.path.join(ROOT, "cvc_b200"), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    return lib


@pytest.fixture(scope="session")
def cb():
    _build_library()
    import cvc_b200
    return cvc_b200


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle_bind
    oracle_bind.build_oracle()
    return oracle_bind


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def seeded(seed, n):
    """Deterministic float64 test data (numpy PCG64 uniforms mapped to [-1, 1))."""
    return np.random.Generator(np.random.PCG64(seed)).random(n) * 2.0 - 1.0


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
