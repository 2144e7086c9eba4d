"""The engine library loads without a GPU and exports every C-ABI symbol
include/nepx.h declares (no compute call is made here)."""
import ctypes
import os
import re

import nepx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nepx.h")).read()
    return sorted(set(re.findall(r"\b(nepx_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(nepx.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(nepx.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_create_rejects_bad_arguments():
    lib = nepx.lib()
    h = ctypes.c_void_p()
    assert lib.nepx_create(None, 10, ctypes.byref(h)) == 1
    assert lib.nepx_create(b"/nonexistent/nep.txt", 0, ctypes.byref(h)) == 1
    assert b"max_atoms" in lib.nepx_last_error(None)
    # the reason of a failed create is kept for this thread (no handle exists)
    assert lib.nepx_create(b"/nonexistent/nep.txt", 10, ctypes.byref(h)) == 2
    msg = lib.nepx_last_error(None)
    assert msg.startswith(b"nepx_create: ") and b"/nonexistent/nep.txt" in msg
