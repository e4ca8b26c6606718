"""Host side of the eye measurements (CPU): the synthetic game frames and the eye layout for the
synthetic connectome that bench.py's eye and fleet components use."""

import numpy as np


def test_game_frames_are_seeded_and_shaped():
    from flyzero_b200 import workloads as wl

    a = wl.game_frames(3, 2, (48, 64), seed=4)
    b = wl.game_frames(3, 2, (48, 64), seed=4)
    c = wl.game_frames(3, 2, (48, 64), seed=5)
    assert a.shape == (2, 3, 48, 64, 3) and a.dtype == np.uint8
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert not np.array_equal(a[0], a[1])                 # the scene moves between frames
    assert not np.array_equal(a[:, 0], a[:, 1])           # every instance has its own scene


def test_eye_layout_for_the_synthetic_drive():
    from flyzero_b200 import workloads as wl

    drive = wl.grating_drive(5000, seed=0, n_inputs=600)
    lo = wl.eye_layout(drive, (224, 256), cell=4, y_min=0.2)
    assert len(lo.idx) == 600 and np.array_equal(lo.idx, drive.inputs)
    assert lo.gx.min() >= 0 and lo.gx.max() < 64 and lo.gy.min() >= 0 and lo.gy.max() < 56
    assert lo.chan.max() < 14 and len(np.unique(lo.chan)) == 14
    np.testing.assert_array_equal(lo.visible, lo.py >= 0.2 * 224)


def test_eye_oracle_runs_the_bench_layout():
    from eye_oracle import EyeOracle
    from flyzero_b200 import workloads as wl

    drive = wl.grating_drive(5000, seed=0, n_inputs=600)
    lo = wl.eye_layout(drive, (224, 256))
    fr = wl.game_frames(1, 3, (224, 256), seed=1)
    o = EyeOracle((224, 256), lo.gx, lo.gy, lo.chan, lo.visible, gain=10 ** 2.7, transient_gain=4.0,
                  sustained_gain=4.0, chromatic_gain=1.0)
    rates = [o.see(f[0]) for f in fr]
    assert all(r.shape == (600,) and r.dtype == np.float32 for r in rates)
    assert np.count_nonzero(rates[2]) > 0 and np.all(rates[2] <= 150.0)
    assert np.all(rates[2][~lo.visible] == 0)
