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
