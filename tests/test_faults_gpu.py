"""Fault drills of the engine, in the forms that fault no GPU: the persistent engine's grid-barrier
wait made to run out (a budget of a few hundred cycles), the spike work lists made to overflow (a
capacity of one item, so items are dropped, never written out of bounds), and bad arguments
through the C ABI. Each drill checks the error code fb_check / the entry point returns, then that
the engine recovers: after fb_reset and the default limits, a run equals that of an engine that
never failed, bit for bit. The reference's only guard on this path is a capacity assert
(flyzero/gpu.py:166-168)."""

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


def _pair(engine, seed=3):
    """Two engines on one network with the same drive: the drilled one and a witness."""
    from flyzero_b200.brain import LIFParams
    from flyzero_b200.gpu import BatchBrain

    conn = cx.synthetic(4096, seed=5)
    idx, rate = wl.config1_inputs(conn.n, seed=5)
    out = []
    for _ in range(2):
        gb = BatchBrain(conn.weights, LIFParams(), batch=4, seed=seed)
        if engine == "persistent" and gb.info().group == 0:
            pytest.skip("persistent engine unavailable")
        gb.set_schedule(engine)
        gb.set_input(idx, rate * 3)
        out.append(gb)
    return out


def _recovers(torch, gb, witness, steps):
    """After the drill: both engines back to rest (same Poisson counter), then identical runs."""
    from flyzero_b200 import _lib

    _lib.check(gb._L.fb_set_limits(gb._h, 0, 0))
    gb.reset()
    witness.reset()
    assert gb.step_no == witness.step_no
    a, b = gb.run_steps(steps).cpu().numpy(), witness.run_steps(steps).cpu().numpy()
    gb.check()
    witness.check()
    assert a.sum() > 0
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(gb.v.cpu().numpy(), witness.v.cpu().numpy())


def test_barrier_wait_runs_out_and_the_engine_recovers(torch):
    from flyzero_b200 import _lib

    gb, witness = _pair("persistent")
    _lib.check(gb._L.fb_set_limits(gb._h, 200, 0))          # 200 cycles: the first barrier times out
    gb.run_steps(40)
    witness.run_steps(40)
    with pytest.raises(_lib.FlyBrainError) as e:
        gb.check()
    assert e.value.code == _lib.FB_ERR_TIMEOUT
    gb.check()                                              # the flags were cleared
    _recovers(torch, gb, witness, 120)


@pytest.mark.parametrize("engine", ["step", "persistent"])
def test_work_list_overflow_is_reported_without_stray_writes(torch, engine):
    from flyzero_b200 import _lib

    gb, witness = _pair(engine)
    cap = int(gb.info().item_capacity)
    assert cap > 1
    gb.reset()
    _lib.check(gb._L.fb_set_limits(gb._h, 0, 1))            # one item per list: the first busy step overflows
    assert int(gb.info().item_capacity) == 1
    gb.run_steps(60)
    witness.run_steps(60)
    with pytest.raises(_lib.FlyBrainError) as e:
        gb.check()
    assert e.value.code == _lib.FB_ERR_OVERFLOW
    _recovers(torch, gb, witness, 120)
    assert int(gb.info().item_capacity) == cap


def test_bad_arguments_through_the_c_abi(torch):
    from flyzero_b200 import _lib
    from flyzero_b200.brain import LIFParams

    L = _lib.load()
    prm = _lib.Params(**{k: float(getattr(LIFParams(), k)) for k, _ in _lib.Params._fields_})
    h = C.c_void_p()

    def create(indptr, indices, data, n):
        indptr = np.asarray(indptr, np.int64)
        indices = np.asarray(indices, np.int32)
        data = np.asarray(data, np.float32)
        return L.fb_create(C.byref(prm), _lib.ptr(indptr, _lib.i64p), _lib.ptr(indices, _lib.i32p),
                           _lib.ptr(data, _lib.f32p), n, len(indices), 2, 0, None, 0, 0, 0, C.byref(h))

    assert create([1, 2, 3], [0, 1], [1, 1], 2) == _lib.FB_ERR_ARG                # indptr must start at 0
    assert "indptr" in _lib.last_error()
    assert create([0, 2, 1], [0, 1], [1, 1], 2) == _lib.FB_ERR_ARG                # decreasing
    assert create([0, 1, 2], [0, 5], [1, 1], 2) == _lib.FB_ERR_ARG                # column out of range
    assert "out of range" in _lib.last_error()
    assert create([0, 2, 2], [1, 1], [1, 1], 2) == _lib.FB_ERR_ARG                # duplicate column
    assert "duplicate" in _lib.last_error()
    assert create([0, 1, 2], [1, 0], [1, 1], 2) == _lib.FB_OK
    try:
        bad = np.array([0, 7], np.int32)                                          # instance 7 of 2
        assert L.fb_reset(h, _lib.ptr(bad, _lib.i32p), 2, None) == _lib.FB_ERR_ARG
        assert "out of range" in _lib.last_error()
        far = np.array([5], np.int64)                                             # neuron 5 of 2
        assert L.fb_set_ext(h, _lib.ptr(far, _lib.i64p), 1) == _lib.FB_ERR_ARG
        assert L.fb_set_limits(h, 0, 1 << 40) == _lib.FB_ERR_ARG                   # above the allocation
        assert L.fb_set_limits(h, -1, 0) == _lib.FB_ERR_ARG
        assert L.fb_set_schedule(h, 9, -1, 0) == _lib.FB_ERR_ARG
        assert L.fb_set_schedule(h, 0, 0, 12) == _lib.FB_ERR_ARG                   # lanes 8/16/32
    finally:
        L.fb_destroy(h)
