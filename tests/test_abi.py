"""The C ABI library: it loads without a GPU, exports every entry point include/*.h declares, and
rejects bad arguments before touching the device."""
import ctypes as C
import os
import re

import pytest

from celv2_b200 import engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in ("celv2_cuda.h", "celv2_pruner.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(celv2_[a-z_0-9]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = engine.library()
    names = declared_functions()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(engine.SIGNATURES), set(names) ^ set(engine.SIGNATURES)


def test_arguments_rejected_before_the_device():
    lib = engine.library()
    h = C.c_void_p()
    assert lib.celv2_create(0, 0, 64, 0, C.byref(h)) == engine.E_INVAL
    assert b"positive" in lib.celv2_last_error()
    assert lib.celv2_create(64, 64, 128, 0, C.byref(h)) == engine.E_INVAL
    assert b"64x64" in lib.celv2_last_error()
    assert lib.celv2_launch(None, None, None, 0, 0, None, -1) == engine.E_INVAL
    assert lib.celv2_kernel_launches(None) == 0


def test_record_layout_matches_header():
    from celv2_b200.records import SB_OUT_DTYPE

    text = open(os.path.join(ROOT, "include", "celv2_decision.h")).read()
    assert "== 38872" in text
    assert SB_OUT_DTYPE.itemsize == 38872
    assert SB_OUT_DTYPE.fields["c_inter_cost"][1] == 3592
    assert SB_OUT_DTYPE.fields["c_rcost"][1] == 15068
