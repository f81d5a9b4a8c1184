"""GPU parity of the NIS gate and outlier refits (cgmli_solver_solve_gated)
with the FP64 oracle's restatement of BackendOptimizer::statisticalGate and the
refit loop of optimizeImpl (src/backend/BackendOptimizer.cpp:394-472,669-686,
1030-1079): the same factors rejected (bit-exact sets), the same passes,
iterations and accepted steps, final states rel 1e-6 and final cost rel 1e-7
(the full-solve bars)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from cgmli_slam_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def gated_pair(oracle, backend, w, iterations, max_refits=3, pre_gate=False, presolve=0):
    x0 = w.state_vector()
    if presolve:
        oracle.lm_solve(w.window, presolve)
    xs = w.state_vector()
    st, rep, g, mask = oracle.lm_solve_gated(w.window, iterations, max_refits=max_refits, pre_gate=pre_gate)
    assert st == 0
    xo = w.state_vector()
    w.set_state_vector(xs)
    s = backend.Solver()
    s.set_windows([w])
    s.solve_gated(iterations, max_refits=max_refits, pre_gate=pre_gate)
    s.synchronize()
    s.read_states()
    gr, gm = s.read_gate(0)
    r = s.reports()[0]
    xg = w.state_vector()
    s.close()
    return (rep, g, mask, xo), (r, gr, gm, xg), xs


@pytest.mark.parametrize("case", ["c1_40", "small_30", "refits_53", "c2_20"])
def test_gated_solve_matches_oracle(oracle, backend, case):
    spec, seed, it = {"c1_40": (synth.C1, 52, 40), "small_30": (replace(synth.C1, keyframes=5, landmarks=200), 52, 30),
                      "refits_53": (replace(synth.C1, landmarks=300), 53, 60), "c2_20": (synth.C2, 58, 20)}[case]
    w = synth.SynthWindow(spec, seed)
    (rep, g, mask, xo), (r, gr, gm, xg), xs = gated_pair(oracle, backend, w, it)
    assert r.status == 0
    assert np.array_equal(gm, mask)
    assert gr.passes == g["passes"] and gr.rejected_total == g["rejected_total"] and gr.rejected_last == g["rejected_last"]
    assert gr.evaluated == g["evaluated"]
    assert r.iterations == rep.iterations and r.accepted_steps == rep.accepted_steps
    assert abs(r.final_cost - rep.final_cost) <= 1e-7 * rep.final_cost
    assert rel(xg - xs, xo - xs) < 1e-6
    assert abs(gr.nis_sum - g["nis_sum"]) <= 1e-7 * g["nis_sum"] and abs(gr.nis_max - g["nis_max"]) <= 1e-7 * g["nis_max"]


def test_pre_gate_at_steady_state(oracle, backend):
    w = synth.SynthWindow(synth.C1, 54)
    (rep, g, mask, xo), (r, gr, gm, xg), xs = gated_pair(oracle, backend, w, 5, pre_gate=True, presolve=10)
    assert g["rejected_pre"] > 0 and gr.rejected_pre == g["rejected_pre"]
    assert np.array_equal(gm, mask)
    assert r.iterations == rep.iterations
    assert rel(xg - xs, xo - xs) < 1e-6


def test_gated_batch_equals_alone(backend):
    """Windows gated in one batch reject the same factors and reach the same
    states as alone (the per-window passes are independent)."""
    windows = synth.make_windows("c4", 4, seed=61)
    x0 = [w.state_vector() for w in windows]
    alone = []
    for w in windows:
        s = backend.Solver()
        s.set_windows([w])
        s.solve_gated(20, pre_gate=False)
        s.synchronize()
        s.read_states()
        alone.append((w.state_vector(), s.read_gate(0)[1]))
        s.close()
    for w, x in zip(windows, x0):
        w.set_state_vector(x)
    s = backend.Solver()
    s.set_windows(windows)
    s.solve_gated(20, pre_gate=False)
    s.synchronize()
    s.read_states()
    for i, (w, x) in enumerate(zip(windows, x0)):
        xa, ma = alone[i]
        assert np.array_equal(s.read_gate(i)[1], ma)
        assert rel(w.state_vector() - x, xa - x) < 1e-8
    assert all(r.status == 0 for r in s.reports())


def test_plain_solve_unchanged_by_gate_fields(oracle, backend):
    """solve() without the gate keeps the reference LM (one pass, no rejection)."""
    w = synth.SynthWindow(synth.C1, 29)
    x0 = w.state_vector()
    st, rep = oracle.lm_solve(w.window, 3)
    xo = w.state_vector()
    w.set_state_vector(x0)
    s = backend.Solver()
    s.set_windows([w])
    s.solve(3)
    s.synchronize()
    s.read_states()
    r = s.reports()[0]
    assert r.iterations == rep.iterations and rel(w.state_vector() - x0, xo - x0) < 1e-6
    g, mask = s.read_gate(0)
    assert g.rejected_total == 0 and mask.sum() == 0


def test_unreachable_threshold_is_the_plain_solve(oracle, backend):
    """A threshold no factor reaches: one pass, nothing rejected, and the plain
    solve's iterations and states."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=200), 59)
    x0 = w.state_vector()
    st, plain = oracle.lm_solve(w.window, 8)
    xo = w.state_vector()
    w.set_state_vector(x0)
    s = backend.Solver()
    s.set_windows([w])
    s.solve_gated(8, nis_threshold=1e300, pre_gate=True)
    s.synchronize()
    s.read_states()
    g, mask = s.read_gate(0)
    r = s.reports()[0]
    assert g.passes == 1 and g.rejected_total == 0 and not mask.any()
    assert r.iterations == plain.iterations
    assert rel(w.state_vector() - x0, xo - x0) < 1e-6
