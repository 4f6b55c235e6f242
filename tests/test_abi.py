"""The C ABI library loads and exports every entry point include/*.h declares
(no GPU needed: nothing here launches work)."""
import ctypes
import glob
import os
import re

import pytest

import poa_b200
import poa_b200.build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(poa_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(poa_b200.LIB_PATH):
        poa_b200.build.build()
    return ctypes.CDLL(poa_b200.LIB_PATH)


def test_header_declares_entry_points():
    names = declared_functions()
    assert "poa_create" in names and "poa_run" in names and "poa_align" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(lib, name):
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_status_strings(lib):
    lib.poa_status_str.restype = ctypes.c_char_p
    assert lib.poa_status_str(0) == b"ok"
    assert lib.poa_status_str(2) == b"backtrack error"


def test_params_defaults_match_cli(lib):
    p = poa_b200._CParams()
    lib.poa_params_init(ctypes.byref(p))
    d = poa_b200.Params()
    for f, _ in poa_b200._CParams._fields_:
        assert getattr(p, f) == int(getattr(d, f)), f


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(poa_b200, "_lib", None)
    monkeypatch.setattr(poa_b200, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        poa_b200.lib()


class _DevWindow(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int32)] + [(f, ctypes.c_void_p) for f in (
        "in_ptr", "in_row", "in_weight", "in_base", "base", "ind", "hq", "hq_loc", "tq", "out_ptr", "out_row")]


@pytest.mark.parametrize("n_rows,qlen,moves_cap,want", [
    (10, 2**31 - 1, 2**31 - 1, 3),          # moves capacity cannot hold n_rows + qlen + 1: POA_BAD_ARG
    (10, 2**31 - 12, 2**31 - 1, 4),         # the query buffer alone exceeds the scratch: POA_OOM
    (2**31 - 8, 1, 2**31 - 1, 4),           # row metadata alone exceeds the scratch: POA_OOM
    (60000, 60000, 2**31 - 1, 4),           # rows x full band far beyond the scratch: POA_OOM
    (10, -1, 100, 3),                       # negative query length: POA_BAD_ARG
])
def test_noalloc_size_checks_never_launch(lib, n_rows, qlen, moves_cap, want):
    """poa_align_noalloc rejects impossible or oversized windows from their
    sizes alone, before it touches the GPU (so this runs without one). The
    pointers are never dereferenced on these paths."""
    lib.poa_align_noalloc.argtypes = [ctypes.POINTER(_DevWindow), ctypes.c_void_p, ctypes.c_int32,
                                      ctypes.POINTER(poa_b200._CParams), ctypes.c_int32, ctypes.c_void_p,
                                      ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    fake = ctypes.c_void_p(0x1000)
    w = _DevWindow(n_rows, *([fake] * 11))
    p = poa_b200._CParams()
    lib.poa_params_init(ctypes.byref(p))
    assert lib.poa_align_noalloc(ctypes.byref(w), fake, qlen, ctypes.byref(p), 0, fake, moves_cap, fake,
                                 None) == want
