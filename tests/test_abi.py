"""The C-ABI library loads and exports every entry point include/clb.h declares."""
import ctypes
import os
import re

import numpy as np
import pytest

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


@pytest.mark.parametrize("change,words", [
    (dict(nx=2), b"too small"),
    (dict(nx=2048, ny=1024, nz=1024), b"2^30"),
    (dict(tau=0.5), b"tau"),
    (dict(n_microbes=99), b"microbe"),
])
def test_create_rejects_bad_domains_before_touching_the_device(clb, change, words):
    """clb_create checks the descriptor on the host and returns CLB_INVALID_ARG with a message;
    none of these reaches a CUDA call (nor reads past the small material array given)."""
    import ctypes as C
    d = clb.DomainDesc()
    d.nx, d.ny, d.nz, d.tau, d.flow_precision, d.ade_precision = 4, 3, 2, 0.8, clb.F32, clb.F32
    d.solid_code, d.bounce_back_code, d.n_pore_codes = 0, 1, 1
    d.pore_codes[0] = 2
    for k, v in change.items():
        setattr(d, k, v)
    mat = np.full(24, 2, dtype=np.int8)
    h = C.c_void_p()
    L = clb.lib()
    assert L.clb_create(C.byref(d), mat.ctypes.data_as(C.c_void_p), C.byref(h)) == 1
    assert not h.value
    assert words in L.clb_global_error()


def test_create_rejects_negative_material_codes(clb):
    import ctypes as C
    d = clb.DomainDesc()
    d.nx, d.ny, d.nz, d.tau = 4, 3, 2, 0.8
    mat = np.full(24, 2, dtype=np.int8)
    mat[7] = -3
    h = C.c_void_p()
    assert clb.lib().clb_create(C.byref(d), mat.ctypes.data_as(C.c_void_p), C.byref(h)) == 1
    assert b"negative" in clb.lib().clb_global_error()
