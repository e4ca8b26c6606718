"""The C-ABI library builds, loads without a GPU and exports every function include/*.h
declares (no compute calls: this runs on CPU)."""

import ctypes as C
import os
import re

from conftest import ROOT


def _declared(headers=("flybrain.h", "flysurrogate.h")):
    names = set()
    for h in headers:
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^\s*int\s+((?:fb|fs)_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_the_boundary():
    names = _declared()
    for must in ("fb_create", "fb_destroy", "fb_run", "fb_reset", "fb_set_ext", "fb_set_plastic",
                 "fb_get_views", "fb_get_info", "fb_set_schedule", "fb_check", "fb_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from flyzero_b200 import _lib

    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_errors_cross_the_boundary_as_codes():
    from flyzero_b200 import _lib

    lib = _lib.load()
    out = C.c_void_p()
    rc = lib.fb_create(None, None, None, None, 0, 0, 0, 0, None, 0, 0, 0, C.byref(out))
    assert rc == _lib.FB_ERR_ARG
    assert "bad connectome arguments" in _lib.last_error()
    assert lib.fb_get_info(None, None) == _lib.FB_ERR_ARG
