"""Shared test set-up: markers, import paths and library builds.

``-m gpu`` tests need a CUDA device and fail (they do not skip) without one;
everything else runs on the CPU.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "distributed-lb-ib_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than ~30 s on the CPU")


def _make(path):
    out = subprocess.run(["make", "-C", path], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError(f"make -C {path} failed:\n{out.stdout[-3000:]}\n{out.stderr[-3000:]}")


@pytest.fixture(scope="session")
def oracle_built():
    _make(os.path.join(ROOT, "oracle"))
    return True


@pytest.fixture(scope="session")
def lbib_built():
    _make(PKG)
    return True


@pytest.fixture(scope="session")
def gpu(lbib_built):
    import lbib
    n = lbib.device_count()
    if n < 1:
        pytest.fail("no CUDA device visible: the -m gpu tests need one", pytrace=False)
    return n
