"""CPU checks of configuration 2's sliding sequence on the oracle: sub-windows
cut from one long trajectory hold the landmarks a sliding window keeps, and a
prior chained through OLD marginalizations lands on the right blocks of the
next window (its reference values are the states it was formed at, with the
keyframe blocks moved down by the keyframe that left)."""
from __future__ import annotations

import numpy as np

from cgmli_slam_b200 import abi, synth


def test_subwindows_keep_the_landmarks_a_sliding_window_keeps():
    long = synth.c2_long_window(3, landmarks=1200)
    for start in (0, 2):
        w = synth.SubWindow(long, start, 10)
        win = w.window
        begin = np.ctypeslib.as_array(win.lm_obs_begin, shape=(w.L + 1,))
        kf = np.ctypeslib.as_array(win.obs_kf, shape=(win.num_observations,))
        akf = np.ctypeslib.as_array(win.lm_anchor_kf, shape=(w.L,))
        assert begin[-1] == win.num_observations and np.all(np.diff(begin) >= 1)
        assert kf.min() >= 0 and kf.max() < 10 and akf.min() >= 0 and akf.max() < 10
        assert win.num_imu == 9


def test_prior_chains_onto_the_next_window(oracle):
    long = synth.c2_long_window(4, landmarks=1200)
    w0 = synth.SubWindow(long, 0, 10)
    st, rep = oracle.lm_solve(w0.window, 3)
    assert st in (0, 8)
    prior = oracle.marginalize_window(w0.window, 0, abi.MARGIN_OLD)
    assert prior["status"] == 0 and prior["rank"] > 0
    w0.store()
    w1 = synth.SubWindow(long, 1, 10)
    w1.set_prior(prior, 1)
    # every keyframe block's reference is the state it was formed at, one keyframe down
    off = 0
    for k, i in zip(w1.prior["kinds"], w1.prior["index"]):
        n = 9 if k == abi.PRIOR_SPEED_BIAS else 1 if k == abi.PRIOR_TIME_OFFSET else 7
        ref = w1.prior["ref"][off:off + n]
        if k == abi.PRIOR_POSE:
            assert np.array_equal(ref, w1.arrays["poses"][7 * i:7 * i + 7])
        elif k == abi.PRIOR_SPEED_BIAS:
            assert np.array_equal(ref, w1.arrays["sb"][9 * i:9 * i + 9])
        off += n
    # the prior's residual at its own reference is r0, so the chained window's cost starts finite
    st, cost = oracle.window_cost(w1.window)
    assert st == 0 and np.isfinite(cost)
    st, rep = oracle.lm_solve(w1.window, 3)
    assert st in (0, 8) and rep.final_cost <= rep.initial_cost
