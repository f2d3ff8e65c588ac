"""The C-ABI library loads and exports every symbol include/hedge_b200.h
declares (no compute calls: runs without a GPU)."""
import ctypes as C
import os
import re

import pytest

from hedge_b200 import _native, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "hedge_b200.h")).read()
    return sorted(set(re.findall(r"\b(hb_[a-z_0-9]+)\s*\(", src)))


def test_library_builds_and_exports_all_symbols():
    build.build()
    lib = _native.load()
    syms = header_symbols()
    assert "hb_rhs" in syms and "hb_lsrk_stage" in syms
    for s in syms:
        assert hasattr(lib, s), s
    assert set(_native.EXPORTED) <= set(syms)


def test_null_arguments_are_rejected_without_touching_the_gpu():
    lib = _native.load()
    h = C.c_void_p()
    assert lib.hb_discr_create(None, C.byref(h)) == _native.HB_ERR_INVALID_ARGUMENT
    assert b"null" in lib.hb_last_error_string()
    assert lib.hb_rhs(None, None, None, None, None, None, None) == _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_rhs_elements(None, 0, 1, None, None, None, None, None, None) == \
        _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_lsrk_stage_elements(None, 0, 1, 0.0, 0.0, 0.0, None, None, None, None, None,
                                      None, None) == _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_lincomb(-1, 0, 1.0, None, 1.0, None, None, None) == \
        _native.HB_ERR_INVALID_ARGUMENT
    assert lib.hb_op_destroy(None) == _native.HB_OK
    desc = _native.hb_discr_desc()
    desc.dim = 4
    assert lib.hb_discr_create(C.byref(desc), C.byref(h)) == _native.HB_ERR_UNSUPPORTED
