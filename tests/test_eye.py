"""The motion eye's host side on CPU: the layout (retinotopy and channels, flyzero/eyes.py:37-87,
flyzero/vision.py:67-124) and the CPU oracle of MotionEye.see (vision.py:136-191), both against
the reference's own outputs in tests/golden/eye.npz."""

import numpy as np
import pytest

import eye_cases as E


@pytest.fixture(scope="module")
def z(golden):
    return golden("eye.npz")


@pytest.mark.parametrize("case", E.cases(), ids=lambda c: c[1])
def test_layout_matches_reference(z, case):
    from flyzero_b200.vision import MotionParams, layout

    k, name, shape, n, kw = case
    lo = layout(E.connectome(z), shape, MotionParams(**kw))
    np.testing.assert_array_equal(lo.idx, z[f"{name}_idx"])
    np.testing.assert_array_equal(lo.px, z[f"{name}_px"])
    np.testing.assert_array_equal(lo.py, z[f"{name}_py"])
    np.testing.assert_array_equal(lo.side, z[f"{name}_side"])


@pytest.mark.parametrize("case", E.cases(), ids=lambda c: c[1])
def test_oracle_matches_reference(z, case):
    from eye_oracle import EyeOracle
    from flyzero_b200.vision import MotionParams, layout

    k, name, shape, n, kw = case
    p = MotionParams(**kw)
    lo = layout(E.connectome(z), shape, p)
    eye = EyeOracle(shape, lo.gx, lo.gy, lo.chan, lo.visible, **E.oracle_params(p))
    fr = E.frames(z, k, name, shape, n)
    got = np.stack([eye.see(f) for f in fr])
    want = z[f"{name}_rates"]
    assert np.count_nonzero(want) > 0
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_layout_needs_motion_neurons(z):
    import pandas as pd
    import scipy.sparse as sp

    from flyzero_b200.connectome import Connectome
    from flyzero_b200.vision import layout

    df = pd.DataFrame(dict(cell_type=["Mi1"] * 5, side=["left"] * 5, pos_x=np.arange(5.0), pos_y=np.arange(5.0),
                           pos_z=np.zeros(5)))
    with pytest.raises(ValueError, match="T4/T5"):
        layout(Connectome(sp.csr_matrix((5, 5), dtype=np.float32), df), (48, 64), __import__(
            "flyzero_b200.vision", fromlist=["MotionParams"]).MotionParams())


def test_eye_params_struct_layout():
    import ctypes as C

    from flyzero_b200._lib import EyeParams

    assert C.sizeof(EyeParams) == 72
    assert EyeParams.gain.offset == 32
