"""The C-ABI library loads and exports every entry point the header declares.

Runs without a GPU: no compute call is made beyond rp_create's device probe,
which must fail loudly (RP_ERR_NOEXT) when no CUDA device is present.
"""
import ctypes as C
import os
import re

import pytest

from romspath_b200 import _lib, build

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "romspath_gpu.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rp_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_expected_api():
    syms = declared_symbols()
    assert set(_lib.EXPORTS) == set(syms), (set(_lib.EXPORTS) ^ set(syms))


def test_library_exports_every_declared_symbol():
    build.build()
    L = C.CDLL(build.LIB)
    for s in declared_symbols():
        assert hasattr(L, s), s


def test_version_string():
    L = _lib.load()
    assert b"sm_100a" in L.rp_version()


def test_create_without_gpu_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    L = _lib.load()
    P = _lib.RpParams()
    P.numpar, P.idt, P.dt, P.deltat, P.sub = 10, 300, 3600, 30.0, 4.0
    G = (_lib.RpGrid * 1)()
    h = C.c_void_p()
    rc = L.rp_create(C.byref(P), 1, G, C.byref(h))
    assert rc == -6  # RP_ERR_NOEXT


def test_null_and_range_arguments_rejected():
    L = _lib.load()
    P = _lib.RpParams()
    h = C.c_void_p()
    assert L.rp_create(None, 1, None, C.byref(h)) == -1
    P.numpar, P.idt, P.dt, P.deltat, P.sub = 10, 300, 3600, 30.0, 4.0
    G = (_lib.RpGrid * 1)()
    assert L.rp_create(C.byref(P), 0, G, C.byref(h)) == -1
    assert L.rp_create(C.byref(P), 6, G, C.byref(h)) == -1
    P.behavior = 4          # the oyster-larva behaviours are outside the implemented path
    assert L.rp_create(C.byref(P), 1, G, C.byref(h)) == -5
    assert L.rp_step(None, None, None, 1, 1, 2, 3) == -1
    assert L.rp_destroy(None) == -1
