"""The C-ABI library builds, loads without a GPU and exports every entry
point include/bsgpu.h declares."""
import ctypes
import os
import re

from bsoft_b200 import build

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bsgpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bsg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header():
    path = build.build()
    lib = ctypes.CDLL(path)
    syms = declared_symbols()
    assert len(syms) >= 10
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_version_and_error_without_device():
    lib = ctypes.CDLL(build.build())
    lib.bsg_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.bsg_version()
