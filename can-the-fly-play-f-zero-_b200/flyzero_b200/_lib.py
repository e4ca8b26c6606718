"""ctypes binding of libflybrain.so (include/flybrain.h) and zero-copy torch views of its buffers.

The engine library is the product: there is no fallback. If the library cannot be loaded, or no
CUDA device is present, every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _build

FB_OK, FB_ERR_ARG, FB_ERR_CUDA, FB_ERR_OVERFLOW, FB_ERR_TIMEOUT, FB_ERR_UNSUPPORTED = range(6)
FB_FLAG_F64, FB_FLAG_ACC_FIXED = 1, 2
FB_ENGINE_AUTO, FB_ENGINE_STEP, FB_ENGINE_PERSISTENT = 0, 1, 2
FB_PROP_PUSH, FB_PROP_PULL = 0, 1

i64p = C.POINTER(C.c_int64)
i32p = C.POINTER(C.c_int32)
u32p = C.POINTER(C.c_uint32)
f32p = C.POINTER(C.c_float)
vp = C.c_void_p


class Params(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("v_rest", "v_reset", "v_th", "tau_m", "tau_syn", "t_ref", "delay",
                                           "w_syn", "f_poisson", "dt")]


class Info(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz", C.c_int64), ("batch", C.c_int32), ("n_delay", C.c_int32),
                ("n_ref", C.c_int32), ("acc_mode", C.c_int32), ("f64", C.c_int32), ("engine", C.c_int32),
                ("propagation", C.c_int32), ("lanes", C.c_int32), ("group", C.c_int32), ("ctas", C.c_int32),
                ("n_plastic", C.c_int64), ("n_ext", C.c_int64), ("t", C.c_int64), ("step_no", C.c_uint32),
                ("launches", C.c_int64), ("item_capacity", C.c_int64), ("bytes_device", C.c_int64),
                ("decay_syn", C.c_double), ("decay_m", C.c_double), ("kick", C.c_double), ("epoch", C.c_int32)]


class Views(C.Structure):
    _fields_ = [("v", vp), ("g", vp), ("ref", vp), ("pw", vp), ("w0", vp), ("ext_idx", vp), ("p_ext", vp),
                ("bias_ext", vp), ("stop_tick", vp)]


class EyeParams(C.Structure):
    _fields_ = [("cell", C.c_int32), ("shift", C.c_int32), ("surround", C.c_int32), ("kernels", C.c_int32),
                ("a_hp", C.c_float),
                ("a_d", C.c_float), ("p_scale", C.c_float), ("gain", C.c_double), ("max_rate", C.c_double),
                ("transient_gain", C.c_double), ("sustained_gain", C.c_double), ("chromatic_gain", C.c_double)]


_LIB = None

# every symbol include/flybrain.h declares, with its signature
SIGNATURES = {
    "fb_create": (C.c_int, [C.POINTER(Params), i64p, i32p, f32p, C.c_int64, C.c_int64, C.c_int32, C.c_uint32,
                            i64p, C.c_int64, C.c_uint32, C.c_int32, C.POINTER(vp)]),
    "fb_destroy": (C.c_int, [vp]),
    "fb_last_error": (C.c_int, [C.c_char_p, C.c_int64]),
    "fb_get_info": (C.c_int, [vp, C.POINTER(Info)]),
    "fb_get_views": (C.c_int, [vp, C.POINTER(Views)]),
    "fb_set_ext": (C.c_int, [vp, i64p, C.c_int64]),
    "fb_set_plastic": (C.c_int, [vp, i64p, C.c_int64]),
    "fb_reset": (C.c_int, [vp, i32p, C.c_int32, vp]),
    "fb_run": (C.c_int, [vp, C.c_int32, vp, vp, vp, vp, vp]),
    "fb_set_schedule": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32]),
    "fb_set_trace": (C.c_int, [vp, vp, C.c_int64]),
    "fb_set_limits": (C.c_int, [vp, C.c_int64, C.c_int64]),
    "fb_trace_rates": (C.c_int, [vp, vp, vp, C.c_int32, vp, C.c_float, C.c_float, vp, C.c_int32, vp, C.c_float,
                                 C.c_float, vp]),
    "fb_delta_apply": (C.c_int, [vp, vp, vp, vp, C.c_int32, vp, C.c_int32, vp, C.c_int32, vp, vp, vp, C.c_int32, vp,
                                 vp, vp]),
    "fb_backprop": (C.c_int, [vp, vp, vp, vp, C.c_int32, vp, C.c_int32, vp, C.c_int32, vp]),
    "fb_eye_state_floats": (C.c_int64, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "fb_motion_eye": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp, vp, vp, vp, C.c_int32, vp, vp, vp, vp, vp, vp, vp]),
    "fb_group_rates": (C.c_int, [vp, vp, vp, vp, C.c_int32, vp, C.c_float, C.c_float, vp, vp]),
    "fb_clamp": (C.c_int, [vp, vp, vp, vp, C.c_int32, vp, vp, C.c_double, C.c_double, C.c_float, C.c_float, vp, vp,
                           vp, vp, vp, vp]),
    "fb_check": (C.c_int, [vp, vp]),
    "fb_reward_step": (C.c_int, [vp, vp, vp, vp, vp, vp, vp, vp, C.c_int32, vp, C.c_double, C.c_double, C.c_float,
                                 C.c_int32, vp]),
    "fb_run_static": (C.c_int, [C.POINTER(Params), C.c_int64, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_uint32,
                                C.c_uint32, C.c_int64, C.c_int32, C.c_int32, vp, vp]),
    # include/flysurrogate.h
    "fs_gemm_kind": (C.c_int, [C.c_int32]),
    "fs_gemm_split": (C.c_int, [C.c_int32]),
    "fs_gemm": (C.c_int, [vp, vp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, vp, vp, vp, vp,
                          vp, C.c_int32, C.c_int32, vp]),
    "fs_poisson_nll": (C.c_int, [vp, vp, C.c_int32, C.c_int32, vp, vp, C.c_int32, vp, vp]),
    "fs_colsum": (C.c_int, [vp, C.c_int32, C.c_int32, C.c_int32, vp, vp]),
    "fs_adam": (C.c_int, [vp, vp, vp, vp, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32, vp, vp,
                          C.c_int32, C.c_int32, C.c_int32, vp]),
    "fs_to_bf16": (C.c_int, [vp, C.c_int64, vp, vp, C.c_int32, C.c_int32, C.c_int32, vp]),
}


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the engine library (building it with nvcc first if it is absent or stale)."""
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if build_if_missing:
            try:
                path = _build.build()
            except Exception as e:  # nvcc missing: fall through to loading what exists
                if not os.path.exists(path):
                    raise RuntimeError(f"flybrain: cannot build {path}: {e}") from e
        if not os.path.exists(path):
            raise RuntimeError(f"flybrain: engine library {path} is missing (build it with flyzero_b200._build)")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().fb_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


class FlyBrainError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"flybrain error {code}: {msg}")
        self.code = code


def check(rc: int):
    if rc != FB_OK:
        raise FlyBrainError(rc, last_error())


def ptr(a: np.ndarray, t):
    return None if a is None else a.ctypes.data_as(t)


class _DeviceArray:
    """An engine-owned device buffer exposed through __cuda_array_interface__ (keeps its owner alive)."""

    def __init__(self, address: int, shape, typestr: str, owner):
        self.__cuda_array_interface__ = {"shape": tuple(int(s) for s in shape), "typestr": typestr,
                                         "data": (int(address), False), "version": 3, "strides": None}
        self._owner = owner


_TYPESTR = {"float32": "<f4", "float64": "<f8", "int8": "|i1", "int32": "<i4", "int64": "<i8"}


def device_tensor(address: int, shape, dtype: str, device, owner):
    import torch

    if int(np.prod(shape)) == 0 or not address:
        return torch.empty(tuple(shape), dtype=getattr(torch, dtype), device=device)
    return torch.as_tensor(_DeviceArray(address, shape, _TYPESTR[dtype], owner), device=device)


class HostStage:
    """Small per-call host arrays copied to the device without blocking the host: a ring of pinned
    buffers, each refilled only after the stream has consumed the copy that last read it (an event
    per buffer). ``put(dst, values)`` enqueues dst <- values on the current stream."""

    def __init__(self, n: int, dtype, slots: int = 4):
        import torch

        self._ring = [[torch.empty(n, dtype=dtype).pin_memory(), None] for _ in range(slots)]
        self._at = 0

    def put(self, dst, values):
        import torch

        buf = self._ring[self._at]
        self._at = (self._at + 1) % len(self._ring)
        if buf[1] is not None:
            buf[1].synchronize()
        buf[0].numpy()[:] = values
        dst.copy_(buf[0], non_blocking=True)
        buf[1] = torch.cuda.Event()
        buf[1].record(torch.cuda.current_stream(dst.device))
