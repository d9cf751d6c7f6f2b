"""The C-ABI library loads and exports every entry point include/bbg.h declares."""
import ctypes
import os
import re

from bulbit_b200 import abi, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "bbg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bbg_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = ctypes.CDLL(lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    bound = {name for name, _, _ in abi.EXPORTS}
    assert set(declared_symbols()) <= bound


def test_struct_sizes_match_header_layout():
    assert ctypes.sizeof(abi.BvhNode) == 32
    assert ctypes.sizeof(abi.Ray) == 32
    assert ctypes.sizeof(abi.Hit) == 16


def test_version_and_error_strings():
    L = lib.get_lib()
    assert b"sm_100a" in L.bbg_version()
    assert L.bbg_bvh_build(None, 0, None, None, None) == abi.BBG_ERR_INVALID_ARG
    assert b"bbg_bvh_build" in L.bbg_last_error()
