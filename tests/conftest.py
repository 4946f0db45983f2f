"""Shared test setup: import paths, the `gpu` marker, reference systems."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pwdft-rs_b200")
for p in (PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

# The oracle's dense eigensolves use BLAS threads; more threads than free
# cores (other jobs on the host) makes spinning BLAS workers crawl.
try:
    from threadpoolctl import threadpool_limits
    threadpool_limits(limits=max(1, min(4, os.cpu_count() or 1)), user_api="blas")
except ImportError:
    pass

GOLDEN = os.path.join(ROOT, "tests", "golden")
UPF_DIR = os.path.join(GOLDEN, "upf")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def upf_path(name):
    return os.path.join(UPF_DIR, name)


@pytest.fixture(scope="session")
def si_pp():
    from pwgpu.upf import load_upf
    return load_upf(upf_path("Si.upf"))


@pytest.fixture(scope="session")
def si_hgh_pp():
    from pwgpu.upf import load_upf
    return load_upf(upf_path("Si_hgh.upf"))


@pytest.fixture(scope="session")
def c_pp():
    from pwgpu.upf import load_upf
    return load_upf(upf_path("C.upf"))


def rng(seed=20261203):
    return np.random.default_rng(seed)
