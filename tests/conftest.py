"""Shared test setup: paths to the package, the oracle and the built library."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "real-time-depth-fusion-directional-tsdf_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libvsg.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def synth_mod():
    import synth

    return synth


@pytest.fixture(scope="session")
def hosttest_lib(tmp_path_factory):
    """Host (gcc) build of the library's header-only helpers, for CPU tests."""
    import ctypes
    import subprocess

    out = str(tmp_path_factory.mktemp("hosttest") / "libvsg_hosttest.so")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", os.path.join(PKG, "csrc"), "-o", out,
                    os.path.join(ROOT, "tests", "hosttest.c"), "-lm"], check=True)
    return ctypes.CDLL(out)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch
