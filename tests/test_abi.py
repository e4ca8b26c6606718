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


def test_static_run_rejects_bad_ticks_and_delays_before_any_device_work():
    """fb_run_static checks its scalar arguments on the host and returns FB_ERR_ARG before it
    touches the device, so these cases run without a GPU (the buffers are never dereferenced)."""
    import math

    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams

    lib = _lib.load()
    buf = (C.c_int64 * 8)()
    b = C.cast(buf, C.c_void_p)

    def call(params, t0=0, steps=1, n=4):
        prm = _lib.Params(**{k: float(getattr(params, k)) for k, _ in _lib.Params._fields_})
        return lib.fb_run_static(C.byref(prm), n, b, b, b, b, b, b, None, None, None, 0, 0, t0, steps, 1, b, None)

    p = LIFParams()
    assert call(p, t0=-1) == _lib.FB_ERR_ARG
    assert "t0" in _lib.last_error()
    assert call(p, t0=2 ** 63 - 1, steps=5) == _lib.FB_ERR_ARG
    for bad in (LIFParams(delay=math.nan), LIFParams(delay=math.inf), LIFParams(delay=1e300),
                LIFParams(delay=-1e300), LIFParams(t_ref=math.nan), LIFParams(t_ref=-5.0), LIFParams(dt=math.inf)):
        assert call(bad) == _lib.FB_ERR_ARG, bad
    # n * (n_delay + 1) beyond the array, including sizes whose product overflows int64
    assert call(p, n=2 ** 40) == _lib.FB_ERR_ARG
    assert "exceeds the static ring" in _lib.last_error()


def test_surrogate_settings_are_checked_on_the_host():
    """fs_gemm_kind / fs_gemm_split only read and set host state: bad values come back as errors
    (fs_gemm_split: -FB_ERR_ARG), good ones return the previous setting."""
    from flyzero_b200 import _lib

    lib = _lib.load()
    old = lib.fs_gemm_split(-1)
    assert 1 <= old <= 8
    assert lib.fs_gemm_split(0) == -_lib.FB_ERR_ARG
    assert lib.fs_gemm_split(9) == -_lib.FB_ERR_ARG
    assert "fs_gemm_split" in _lib.last_error()
    assert lib.fs_gemm_split(3) == old
    assert lib.fs_gemm_split(old) == 3
    kind = lib.fs_gemm_kind(-1)
    assert lib.fs_gemm_kind(7) == _lib.FB_ERR_ARG
    assert lib.fs_gemm_kind(-1) == kind
