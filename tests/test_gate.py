"""CPU tests of the oracle's NIS gate and outlier refits
(BackendOptimizer::statisticalGate and the refit loop of optimizeImpl,
src/backend/BackendOptimizer.cpp:394-472,669-686,1030-1079)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from cgmli_slam_b200 import abi, synth

NIS = 9.210340371976184  # visualNisThreshold (src/backend/BackendTypes.hpp:186)


def test_gate_rejects_planted_outliers(oracle):
    w = synth.SynthWindow(synth.C1, 51)
    planted = w.outliers().astype(bool)
    st, rep, g, mask = oracle.lm_solve_gated(w.window, 10, pre_gate=False)
    assert st == 0
    m = mask.astype(bool)
    assert np.all(m[planted])  # every gross outlier is gated out
    assert g["rejected_total"] == m.sum() and g["passes"] >= 1
    assert g["evaluated"] == w.F  # the first post-solve gate saw every factor


def test_refits_share_the_iteration_budget(oracle):
    spec = replace(synth.C1, keyframes=5, landmarks=200)
    for max_refits in (0, 1, 3):
        w = synth.SynthWindow(spec, 52)
        st, rep, g, mask = oracle.lm_solve_gated(w.window, 30, max_refits=max_refits, pre_gate=False)
        assert st == 0
        assert rep.iterations <= 30
        assert 1 <= g["passes"] <= max_refits + 1
        if g["passes"] < max_refits + 1 and rep.iterations < 30:
            assert g["rejected_last"] == 0  # stopped because the last gate was clean
    # with refits left and a clean last gate, every evaluated energy is under the threshold
    w = synth.SynthWindow(replace(synth.C1, landmarks=300), 53)
    st, rep, g, mask = oracle.lm_solve_gated(w.window, 60, max_refits=3, pre_gate=False)
    assert st == 0 and g["passes"] == 4 and rep.iterations < 60 and g["rejected_last"] == 0
    assert g["nis_max"] <= NIS


def test_pre_gate_at_steady_state(oracle):
    """Gated solve of an already solved window: the pre-solve gate removes the
    factors above the threshold at the current states before the first pass."""
    w = synth.SynthWindow(synth.C1, 54)
    oracle.lm_solve(w.window, 10)
    st, rep, g, mask = oracle.lm_solve_gated(w.window, 5, pre_gate=True)
    assert st == 0 and g["rejected_pre"] > 0
    assert g["rejected_total"] >= g["rejected_pre"]
    assert mask.sum() == g["rejected_total"]


def test_rejected_factors_leave_the_problem(oracle):
    """A gated factor contributes nothing afterwards: the window's cost with the
    rejected whitening rows zeroed equals the solve's final cost."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=200), 57)
    st, rep, g, mask = oracle.lm_solve_gated(w.window, 60, max_refits=3, pre_gate=False)
    # a clean last gate: every rejection happened before the final pass's cost
    assert st == 0 and g["passes"] == 3 and g["rejected_last"] == 0
    Pz = np.ctypeslib.as_array(w.window.obs_P, shape=(6 * w.F,)).reshape(-1, 6).copy()
    Pz[mask.astype(bool)] = 0.0
    Pz = np.ascontiguousarray(Pz.ravel())
    win = abi.Window.from_buffer_copy(w.window)
    win.obs_P = Pz.ctypes.data_as(abi.c_double_p)
    s2, cost = oracle.window_cost(win)
    assert s2 == 0 and abs(cost - rep.final_cost) <= 1e-9 * rep.final_cost
