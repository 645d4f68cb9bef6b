"""The C-ABI library loads and exports every entry point include/clb.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "clb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(clb_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported(clb):
    L = ctypes.CDLL(clb.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(clb):
    assert set(declared_symbols()) <= set(clb.SIGNATURES)


def test_null_arguments_return_status_not_crash(clb):
    L = clb.lib()
    assert L.clb_create(None, None, None) == 1
    assert b"null" in L.clb_global_error()
    assert L.clb_flow_step(None, 1) == 1
