"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ensure_oracle():
    lib = ROOT / "oracle" / "liboracle.so"
    if not lib.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), str(lib)], check=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle()
    from oracle import cpu
    return cpu


@pytest.fixture(scope="session")
def conan():
    import conan_b200
    return conan_b200


@pytest.fixture(scope="session")
def gpu(conan):
    import ctypes
    n = ctypes.c_int()
    conan._lib.lib().conan_device_count(ctypes.byref(n))
    if n.value < 1:
        pytest.fail("no CUDA device visible to libconan_pm.so")
    return 0


def load_golden(name):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
