"""Host logic of the schedule autotuner (no GPU)."""

import pytest

from flyzero_b200.gpu import choose_schedule


def test_choose_schedule_picks_the_fastest():
    t = {("persistent", "push", 8): 0.012, ("step", "push", 8): 0.030, ("step", "pull", 8): 0.5}
    assert choose_schedule(t) == ("persistent", "push", 8)
    t[("step", "pull", 8)] = 0.001
    assert choose_schedule(t) == ("step", "pull", 8)


def test_choose_schedule_ties_keep_the_first_listed():
    t = {("step", "push", 32): 1.0, ("step", "push", 8): 1.0}
    assert choose_schedule(t) == ("step", "push", 32)


def test_choose_schedule_needs_a_timing():
    with pytest.raises(ValueError):
        choose_schedule({})
