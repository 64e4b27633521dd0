"""The C-ABI library loads and exports every function include/wigner_b200.h declares."""
import ctypes
import os
import re

import pytest

from pywignercuda2_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "wigner_b200.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "while", "defined")))


def test_header_declares_entry_points():
    names = declared()
    for must in ("wig_faft", "FAFT64_4D_Z2Z", "wig4d_plan_create", "wig4d_run", "wig4d_reduce"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_signatures_cover_header():
    names = declared()
    missing = [n for n in names if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_status_strings_without_gpu():
    lib = _lib.load()
    assert lib.wig_status_string(0) == b"ok"
    assert lib.wig_version() >= 100


def test_invalid_arguments_rejected_on_host():
    """Argument checks run before any CUDA call, so they work without a GPU."""
    lib = _lib.load()
    shape = (ctypes.c_int * 4)(4, 4, 4, 4)
    assert lib.wig_faft(None, shape, 0, 1, 0.1, 0.25, 1.0, None) == 1
    assert lib.wig_faft(ctypes.c_void_p(16), shape, 0, 7, 0.1, 0.25, 1.0, None) == 1
    assert lib.wig_faft(ctypes.c_void_p(16), shape, 9, 1, 0.1, 0.25, 1.0, None) == 1
    assert lib.wig4d_plan_create(None, None) == 1
    assert lib.wig4d_run(None, None, 1, None, None) == 1
    assert lib.FAFT64_4D_Z2Z(ctypes.c_void_p(16), 0.1, 0.1, 1, 0, 1.0) == 2   # segment != 0
