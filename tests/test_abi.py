"""The C-ABI library loads and exports every entry point include/sailfish_b200.h declares;
argument checks that need no GPU behave as documented."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "sailfish_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sf_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "sf_ctx_create" in syms and "sf_rhs3d" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol():
    from sailfish_b200 import _lib
    for s in declared_symbols():
        assert hasattr(_lib.lib, s), s
        assert s in _lib.SIGNATURES, "no ctypes signature for %s" % s


def test_version_and_argument_errors():
    from sailfish_b200 import _lib
    L = _lib.lib
    assert L.sf_version() == 1
    out = ctypes.c_void_p()
    assert L.sf_ctx_create(None, ctypes.byref(out)) == _lib.SF_EINVAL
    d = _lib.GridDesc()
    d.L, d.M, d.N, d.precision = 10, 10, 6, 7
    assert L.sf_ctx_create(ctypes.byref(d), ctypes.byref(out)) == _lib.SF_EDTYPE
    assert b"precision" in L.sf_last_error()
    d.precision = _lib.SF_FP32
    d.N = 3
    assert L.sf_ctx_create(ctypes.byref(d), ctypes.byref(out)) == _lib.SF_EINVAL
    assert L.sf_rhs3d(None, *([None] * 9)) == _lib.SF_EINVAL
    assert L.sf_ctx_destroy(None) == _lib.SF_OK


def declared_arity():
    """name -> number of parameters of each prototype in the header."""
    with open(os.path.join(ROOT, "include", "sailfish_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for name, params in re.findall(r"\b(sf_[a-z0-9_]+)\s*\(([^()]*)\)\s*;", text):
        params = params.strip()
        out[name] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_signatures_match_the_header_arity():
    """Each ctypes signature has as many arguments as the header's prototype (a missing or extra
    argument would shift every later one)."""
    from sailfish_b200 import _lib
    arity = declared_arity()
    assert len(arity) >= 20
    for name, n in arity.items():
        assert len(_lib.SIGNATURES[name]) == n, (name, len(_lib.SIGNATURES[name]), n)
