"""Test configuration.

Markers: `gpu` tests need a CUDA device and the built CUDA library; everything
else runs on the CPU.  The CPU restatement (oracle/) is built on demand and is
used only as the checker.
"""
import ctypes as C
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "liborc.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and libscfd_b200.so")


def build_oracle():
    srcs = [os.path.join(ROOT, "oracle", f) for f in ("oracle.cpp", "cea.cpp", "dvode.h", "Makefile")]
    srcs.append(os.path.join(ROOT, "include", "scfd_b200.h"))
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < max(os.path.getmtime(s) for s in srcs):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    return ORACLE_SO


@pytest.fixture(scope="session")
def orc():
    from shared_cfd_b200 import abi
    return abi.Bound(C.CDLL(build_oracle()), "orc_")


@pytest.fixture(scope="session")
def orc_raw():
    return C.CDLL(build_oracle())


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from shared_cfd_b200 import build, solver
    build.build()
    return solver.load_library()


# A checkout of the reference (ISASShimadaLab/shared_cfd) for the tests that read
# its sample files directly; those tests are skipped when SCFD_REFERENCE is unset.
REFERENCE = os.environ.get("SCFD_REFERENCE", "")
