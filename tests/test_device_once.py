"""CPU test of the once-per-device set-up helper (nqpu_b200/csrc/device_once.h),
which replaces process-wide "configured" flags for kernel attributes and the
per-device SM count: concurrent host threads, several device indices, each
device's set-up run exactly once."""
import ctypes as C
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
SRC = ROOT / "tests" / "device_once_check.cpp"
HDR = ROOT / "nqpu_b200" / "csrc" / "device_once.h"
SO = ROOT / "tests" / "_build" / "libdeviceonce.so"


@pytest.fixture(scope="module")
def check():
    SO.parent.mkdir(exist_ok=True)
    if not SO.exists() or SO.stat().st_mtime < max(SRC.stat().st_mtime, HDR.stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-pthread", "-I",
                        str(ROOT / "nqpu_b200" / "csrc"), str(SRC), "-o", str(SO)], check=True)
    lib = C.CDLL(str(SO))
    lib.per_device_once_check.restype = C.c_int
    lib.per_device_once_check.argtypes = [C.c_int, C.c_int, C.c_int]
    return lib.per_device_once_check


@pytest.mark.parametrize("threads,devices", [(1, 1), (8, 1), (16, 3), (32, 8), (4, 64)])
def test_setup_runs_once_per_device(check, threads, devices):
    assert check(threads, devices, 200) == 0
