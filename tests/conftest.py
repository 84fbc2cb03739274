"""Shared test setup: import paths, the `gpu` marker, and in-tree builds.

Tests marked ``gpu`` need a B200 and call libmfgpu through its C ABI; the
rest run on the CPU (oracle against its golden vectors, host symbolic code,
ABI exports, multi-process host logic).
"""

import ctypes
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pureumfpack.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _ensure_built():
    """Rebuild libmfgpu.so when any of its sources or headers is newer than
    the library (build.up_to_date compares them), and the oracle through its
    Makefile, so the tests never run a stale binary."""
    import build

    build.build()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def emu(tmp_path_factory):
    """tests/plan_emulator.cpp with the library's plan and symbolic sources:
    the device factorization's semantics run over the library's own Plan on
    the CPU."""
    here = os.path.dirname(os.path.abspath(__file__))
    csrc = os.path.join(PKG, "csrc")
    out = str(tmp_path_factory.mktemp("emu") / "libplanemu.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", csrc, "-o", out,
                    os.path.join(here, "plan_emulator.cpp"), os.path.join(csrc, "plan.cpp"),
                    os.path.join(csrc, "host", "symbolic.cpp"), "-lpthread"], check=True)
    return ctypes.CDLL(out)
