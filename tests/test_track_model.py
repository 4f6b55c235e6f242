"""The batch kernel's one-pass record choices against the reference-shaped
per-predecessor tests, on the CPU.

The adaptive batch fill folds every predecessor's terms into running maxima
and first-position fields while it reads the predecessors once
(dp_core.h track_d / track_m / track_record). tests/model/track_check.cpp
runs that formulation next to flags_pred + encode_wide (the comparisons of
the reference's backtrack, src/align.cpp:1592-1604 and 1632-1658, pinned by
the golden cases through the CPU model) on random blocks with many ties and
requires identical 4-byte records wherever the kernel uses the one-pass form.
"""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "model", "build", "libtrack_check.so")


@pytest.fixture(scope="module")
def lib():
    src = os.path.join(HERE, "model", "track_check.cpp")
    hdr = os.path.join(ROOT, "poa_b200", "csrc", "dp_core.h")
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not os.path.exists(LIB) or max(os.path.getmtime(src), os.path.getmtime(hdr)) > os.path.getmtime(LIB):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                        "-I" + os.path.join(ROOT, "poa_b200", "csrc"), src, "-o", LIB], check=True)
    L = ctypes.CDLL(LIB)
    L.track_check.restype = ctypes.c_int
    L.track_check.argtypes = [ctypes.c_uint64, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    return L


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_one_pass_choices_match_reference_tests(lib, seed):
    n = ctypes.c_int()
    bad = lib.track_check(seed, 50000, ctypes.byref(n))
    assert n.value > 50000  # cells compared
    assert bad == 0
