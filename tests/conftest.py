"""Shared pytest setup.

* ``gpu`` marker: tests that need a B200 (run with ``-m gpu``).
* The reference AVX library asserts on more than 32 OpenMP threads
  (reg.avx.cpp:7,103), so OMP_NUM_THREADS is capped before any OpenMP
  runtime is initialised.
* ``nb6b200`` (the product package) and ``oracle`` (test infrastructure) are
  put on sys.path.
"""
import os
import sys

_ncpu = os.cpu_count() or 1
os.environ.setdefault("OMP_NUM_THREADS", str(min(32, _ncpu)))

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nbody6ppgpu-beijing_b200")
for p in (PKG, ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import pytest  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAVE_GPU = _have_gpu()


def pytest_collection_modifyitems(config, items):
    if HAVE_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def nb6():
    """The product library (libnb6b200.so) through the reference-ABI mirror."""
    import nb6b200
    lib = nb6b200.load()
    return lib


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle
