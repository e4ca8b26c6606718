"""fb_run_static, the entry point for callers that cannot allocate device memory at run time
(their GPU memory belongs to another allocator's pool, or an allocation's implicit device
synchronisation is not acceptable mid-run, or run-time allocation is forbidden after start-up).

It keeps its only scratch, the synaptic input in flight, in an array compiled into the library, so
its output must equal that of the allocating entry point (fb_run through BatchBrain, Q32.32 mode)
bit for bit, over two calls in a row that continue one simulation through that array. Collected
last on purpose: it may run alone in a fresh process or after every other test."""

import ctypes as C

import numpy as np
import pytest

from flyzero_b200 import connectome as cx
from flyzero_b200 import workloads as wl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _params(p):
    from flyzero_b200 import _lib

    return _lib.Params(**{k: float(getattr(p, k)) for k, _ in _lib.Params._fields_})


def test_static_run_matches_allocating_entry_point(torch):
    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    L = _lib.load()
    p = LIFParams()
    conn = cx.synthetic(8192, seed=4)
    n = conn.n
    idx, rate = wl.config1_inputs(n, seed=4)
    gb = BatchBrain(conn.weights, p, batch=1, seed=9, fixed_point=True)
    assert gb.info().acc_mode == 1
    gb.set_input(idx, rate * 3)
    gb.set_bias(idx[:5], 3.0)
    dev = gb.device
    # caller-owned buffers of the allocation-free path
    indptr = torch.as_tensor(gb.indptr, device=dev)
    indices = torch.as_tensor(gb.indices, device=dev)
    weights = torch.as_tensor(gb.data, device=dev)
    v = torch.full((n,), p.v_rest, dtype=torch.float32, device=dev)
    g = torch.zeros(n, dtype=torch.float32, device=dev)
    ref = torch.zeros(n, dtype=torch.int8, device=dev)
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    prm = _params(p)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    steps = 400
    for call in range(2):
        free_before = torch.cuda.mem_get_info(dev)[0]
        rc = L.fb_run_static(C.byref(prm), n, _ptr(indptr), _ptr(indices), _ptr(weights), _ptr(v), _ptr(g),
                             _ptr(ref), _ptr(gb.d_ext_idx), _ptr(gb.p_ext), _ptr(gb.bias_ext), 9, call * steps,
                             call * steps, steps, 1 if call == 0 else 0, _ptr(counts), stream)
        assert rc == _lib.FB_OK, _lib.last_error()
        torch.cuda.synchronize(dev)
        if call == 1:     # the first call on a device may load the module that holds the array
            assert torch.cuda.mem_get_info(dev)[0] == free_before, "fb_run_static allocated device memory"
        want = gb.run_steps(steps)[0]
        torch.cuda.synchronize(dev)
        assert int(want.sum()) > 0
        assert torch.equal(counts, want), f"call {call}: spike counts differ"
        assert torch.equal(v, gb.v[0]) and torch.equal(g, gb.g[0]) and torch.equal(ref, gb.ref[0]), \
            f"call {call}: state differs"


def test_static_run_rejects_networks_beyond_its_array(torch):
    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams

    L = _lib.load()
    p = LIFParams()                       # n_delay 18: the ring holds n * 19 entries
    n = _lib_limit(L) // 19 + 1
    dev = torch.device("cuda", torch.cuda.current_device())
    z64 = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    z32 = torch.zeros(n, dtype=torch.int32, device=dev)
    zf = torch.zeros(n, dtype=torch.float32, device=dev)
    z8 = torch.zeros(n, dtype=torch.int8, device=dev)
    rc = L.fb_run_static(C.byref(_params(p)), n, _ptr(z64), _ptr(z32), _ptr(zf), _ptr(zf), _ptr(zf), _ptr(z8),
                         None, None, None, 0, 0, 0, 1, 1, _ptr(z32), None)
    assert rc == _lib.FB_ERR_ARG
    assert "exceeds the static ring" in _lib.last_error()


def _lib_limit(L):
    import os
    import re

    from conftest import ROOT

    text = open(os.path.join(ROOT, "include", "flybrain.h")).read()
    return int(re.search(r"#define FB_STATIC_RING_ENTRIES (\d+)", text).group(1))


def _static_vs_engine(torch, conn, p, steps, with_inputs):
    """Run one instance through fb_run_static and through BatchBrain (Q32.32 mode) and compare."""
    from flyzero_b200 import _lib
    from flyzero_b200.gpu import BatchBrain

    L = _lib.load()
    n = conn.n
    gb = BatchBrain(conn.weights, p, batch=1, seed=9, fixed_point=True)
    if with_inputs:
        idx, rate = wl.config1_inputs(n, seed=4)
        gb.set_input(idx, rate * 3)
    else:                                   # no ext slots: a depolarised, seeded start makes the net fire
        gen = torch.Generator(device=gb.device).manual_seed(5)
        gb.v.copy_(torch.rand(gb.v.shape, generator=gen, device=gb.device) * 8.0 + p.v_rest)
        gb.g.copy_(torch.rand(gb.g.shape, generator=gen, device=gb.device) * 10.0)
    dev = gb.device
    indptr = torch.as_tensor(gb.indptr, device=dev)
    indices = torch.as_tensor(gb.indices, device=dev)
    weights = torch.as_tensor(gb.data, device=dev)
    v, g, ref = gb.v[0].clone(), gb.g[0].clone(), gb.ref[0].clone()
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    ext = (_ptr(gb.d_ext_idx), _ptr(gb.p_ext), _ptr(gb.bias_ext)) if with_inputs else (None, None, None)
    for call in range(2):
        rc = L.fb_run_static(C.byref(_params(p)), n, _ptr(indptr), _ptr(indices), _ptr(weights), _ptr(v), _ptr(g),
                             _ptr(ref), *ext, 9, call * steps, call * steps, steps, 1 if call == 0 else 0,
                             _ptr(counts), stream)
        assert rc == _lib.FB_OK, _lib.last_error()
        want = gb.run_steps(steps)[0]
        torch.cuda.synchronize(dev)
        if call == 0:
            assert int(want.sum()) > 0
        assert torch.equal(counts, want), f"call {call}: spike counts differ"
        assert torch.equal(v, gb.v[0]) and torch.equal(g, gb.g[0]) and torch.equal(ref, gb.ref[0]), \
            f"call {call}: state differs"


def test_static_run_without_ext_inputs(torch):
    from flyzero_b200.brain import LIFParams

    _static_vs_engine(torch, cx.synthetic(4096, seed=6), LIFParams(), 150, with_inputs=False)


def test_static_run_at_the_exact_array_limit(torch):
    """n * (n_delay + 1) equal to the array's size: 65,536 neurons with a 1.5 ms delay (16 slots)."""
    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams

    p = LIFParams(delay=1.5)
    n = _lib_limit(_lib.load()) // 16
    assert n == 65536 and max(1, round(p.delay / p.dt)) + 1 == 16
    _static_vs_engine(torch, cx.synthetic(n, seed=8), p, 120, with_inputs=True)
