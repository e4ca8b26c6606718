"""Host logic of the persistent engine's phase trace: phase_summary turns the per-step, per-CTA
clock stamps (slot order of the kernel's trace) into median phase times. Checked on a synthetic
trace whose phases have known lengths."""

import numpy as np

from flyzero_b200.gpu import TRACE_SLOTS, phase_summary


def _trace(steps=12, ctas=5, K=4, mhz=2000.0):
    """Stamps in SM cycles: kicks 2 us, wait 0.5 us, loop 4 us (CTA c: +0.1 c us), 0.5 us to the
    next step; listing 3 us; push 10 us at each epoch's first step; barrier 1.5 us at its last."""
    T = np.zeros((steps, ctas, TRACE_SLOTS), np.int64)
    us = lambda x: int(round(x * mhz))
    for c in range(ctas):
        t = 1000.0
        for s in range(steps):
            loop = 4.0 + 0.1 * c
            T[s, c, 0] = us(t)
            T[s, c, 4] = us(t + 2.0)
            T[s, c, 1] = us(t + 2.0)
            T[s, c, 2] = us(t + 2.5)
            T[s, c, 3] = us(t + 2.5 + loop)
            T[s, c, 8] = us(t + 3.0)
            if s % K == 0:
                T[s, c, 7], T[s, c, 10] = us(t), us(t + 10.0)
            end = t + 2.5 + loop + 0.5
            if s % K == K - 1:
                T[s, c, 5], T[s, c, 6] = us(end), us(end + 1.5)
                end += 1.5
            t = end
    return T, K, mhz


def test_phase_summary_recovers_the_phase_lengths():
    T, K, mhz = _trace()
    ph = phase_summary(T, K, mhz)
    assert abs(ph["start_to_kicks_drawn"] - 2.0) < 1e-6
    assert abs(ph["slice_wait"] - 0.5) < 1e-6
    assert abs(ph["neuron_loop"] - 4.2) < 1e-6                 # the median CTA (c = 2)
    assert abs(ph["neuron_loop_max_over_ctas"] - 4.4) < 1e-6
    assert abs(ph["listing"] - 3.0) < 1e-6
    assert abs(ph["push_per_epoch"] - 10.0) < 1e-6
    assert abs(ph["grid_barrier_wait"] - 1.5) < 1e-6
    # most steps end 0.5 us after the loop; over all steps and CTAs (plain steps 7.0-7.4 us, the
    # epochs' last steps 1.5 us longer) the median step is 7.3 us
    assert abs(ph["loop_end_to_next_step"] - 0.5) < 1e-6
    assert abs(ph["step"] - 7.3) < 1e-6
