"""Deterministic sums (cgmli_tuning.deterministic = 1): bitwise-reproducible windows.

With FP64 atomics the J^T J pass and the Schur pass add their work units into a
window's sums in an order set by scheduling, so a window's result is the same alone
and in a batch, or eager and replayed, only to rounding (1e-8 after 5 iterations;
the reference's own accumulation, src/backend/VisualCudaBatch.cu:85-93, has the same
property).  In deterministic mode each window's units sum into slots of their own and
one reduction adds the slots in unit order: the tests below require equality of every
bit, and the same S, rhs and step as the atomic form at the parity bars.
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


def _solve(backend, windows, iterations, precision, det=1, tuning=None):
    s = backend.Solver(precision=precision)
    t = dict(tuning or {})
    t["deterministic"] = det
    s.set_tuning(**t)
    s.set_windows(windows)
    s.solve(iterations)
    s.synchronize()
    s.read_states()
    reports = [(r.iterations, r.accepted_steps, r.status, r.final_cost, r.lambda_) for r in s.reports()]
    s.close()
    return [w.state_vector().copy() for w in windows], reports


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_batch_equals_alone_bitwise(backend, precision):
    """Six windows of the batched workload, 5 LM iterations: each window's states and
    report are bit for bit the same solved alone and inside the batch."""
    windows = synth.make_windows("c4", 6, seed=77)
    x0 = [w.state_vector().copy() for w in windows]
    alone = []
    for w in windows:
        states, reports = _solve(backend, [w], 5, precision)
        alone.append((states[0], reports[0]))
    for w, x in zip(windows, x0):
        w.set_state_vector(x)
    states, reports = _solve(backend, windows, 5, precision)
    for (a, ra), b, rb in zip(alone, states, reports):
        assert np.array_equal(a, b)
        assert ra == rb
    assert all(r[2] == 0 for r in reports)


def test_wide_window_in_a_batch_equals_alone_bitwise(backend):
    """A wide window (457 retained columns: the multi-CTA factorization, more Schur
    chunks than units) next to a narrow one, 3 iterations: bitwise the same as alone,
    and any batch order gives the same bits."""
    wide = synth.SynthWindow(replace(synth.C3, landmarks=4000), 3)
    narrow = synth.SynthWindow(synth.C1, 4)
    x0 = [wide.state_vector().copy(), narrow.state_vector().copy()]
    a, ra = _solve(backend, [wide], 3, abi.PRECISION_FP64)
    wide.set_state_vector(x0[0])
    b, rb = _solve(backend, [narrow, wide], 3, abi.PRECISION_FP64)
    nb = b[0].copy()
    assert np.array_equal(a[0], b[1]) and ra[0] == rb[1]
    wide.set_state_vector(x0[0])
    narrow.set_state_vector(x0[1])
    c, rc = _solve(backend, [wide, narrow], 3, abi.PRECISION_FP64)
    assert np.array_equal(c[0], a[0]) and np.array_equal(c[1], nb) and rc[1] == rb[0]


def test_repeat_and_graph_replay_are_bitwise(backend):
    """Five LM iterations, eager, captured and replayed as a CUDA graph, and with the
    per-kernel timing hooks: every run gives the same bits and the same launch count
    (with atomics only one iteration stays at rounding level)."""
    windows = synth.make_windows("c4", 8, seed=61)
    s = backend.Solver()
    s.set_tuning(deterministic=1)
    s.set_windows(windows)
    s.checkpoint()
    results = []
    for mode in ("eager", "capture", "replay", "replay", "profiled"):
        s.rollback()
        if mode == "profiled":
            s.kernel_times(enable=1)
        s.solve(5)
        s.synchronize()
        launches = s.timing()[1]
        if mode == "profiled":
            s.kernel_times(enable=0)
        s.read_states()
        results.append(([w.state_vector().copy() for w in windows],
                        [(r.iterations, r.accepted_steps, r.status, r.final_cost) for r in s.reports()], launches))
    s.close()
    base_states, base_reports, base_launches = results[0]
    for states, reports, launches in results[1:]:
        assert reports == base_reports and launches == base_launches
        for a, b in zip(states, base_states):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_same_system_and_step_as_the_atomic_form(backend, precision):
    """Only the order of additions differs from the atomic form: the reduced system at
    the parity bar of the oracle tests (rel 1e-12), the step at 1e-9, and 5 iterations
    to the same accepted steps with states within 1e-7 (5 iterations amplify a
    rounding-level difference in a weakly constrained window to about 1e-8..1e-7; the
    LM parity bar against the oracle is 1e-6)."""
    windows = synth.make_windows("c4", 5, seed=83) + [synth.SynthWindow(replace(synth.C3, keyframes=20, landmarks=1500), 5)]
    x0 = [w.state_vector().copy() for w in windows]
    solvers = []
    for det in (0, 1):
        s = backend.Solver(precision=precision)
        s.set_tuning(deterministic=det)
        s.set_windows(windows)
        s.step(1e-4)
        s.synchronize()
        solvers.append(s)
    for i in range(len(windows)):
        Sa, ra = solvers[0].read_reduced(i)
        Sd, rd = solvers[1].read_reduced(i)
        assert rel(Sd, Sa) < 1e-12 and rel(rd, ra) < 1e-12
        assert rel(solvers[1].read_step(i)["delta"], solvers[0].read_step(i)["delta"]) < 1e-9
    for s in solvers:
        s.close()
    runs = []
    for det in (0, 1):
        for w, x in zip(windows, x0):
            w.set_state_vector(x)
        runs.append(_solve(backend, windows, 5, precision, det=det))
    (sa, ra), (sd, rd) = runs
    for a, b, x in zip(sa, sd, x0):
        assert rel(b - x, a - x) < 1e-7
    assert [r[:3] for r in ra] == [r[:3] for r in rd]


def test_autotune_keeps_deterministic(backend):
    windows = synth.make_windows("c4", 8, seed=89)
    s = backend.Solver()
    s.set_tuning(deterministic=1)
    best = s.autotune(windows, 1)
    assert best["deterministic"] == 1 and s.get_tuning()["deterministic"] == 1
    s.close()
