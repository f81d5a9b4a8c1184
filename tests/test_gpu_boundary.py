"""The boundary options on the device against the oracle, through the C ABI:
solve-time charts (constant blocks, bias-frozen speed/bias, rotation-only and
fixed extrinsics, held landmarks; BackendOptimizer.cpp:44-91,783-795), the
time budget with minimum iterations (:177,242), caller-evaluated factors
(solveOnline's retainedH / retainedG, VisualCudaBatch.hpp:61,
BackendOptimizer.cpp:210-225), and the device-memory accounting of the solver
and the server."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from boundary_cases import PriorAsHostFactor, set_charts, without_prior
from cgmli_slam_b200 import abi, synth

pytestmark = pytest.mark.gpu

SPEC = replace(synth.C2, landmarks=400)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


def _charted(seed, kind, spec=SPEC):
    w = synth.SynthWindow(spec, seed)
    K, E, L = w.K, w.window.num_extrinsics, w.L
    if kind == "constant":
        kf = np.zeros(K, np.uint8)
        kf[0] = abi.FIX_POSE | abi.FIX_VELOCITY | abi.FIX_BIAS
        ext = np.zeros(E, np.uint8)
        ext[2] = abi.CHART_FIXED
        set_charts(w, kf_fixed=kf, ext_chart=ext)
    elif kind == "scoped":  # latest two poses and velocities free, biases frozen, the rest constant
        kf = np.full(K, abi.FIX_POSE | abi.FIX_VELOCITY | abi.FIX_BIAS, np.uint8)
        kf[-2:] = abi.FIX_BIAS
        set_charts(w, kf_fixed=kf, ext_chart=np.full(E, abi.CHART_FIXED, np.uint8))
    elif kind == "rotation":
        ext = np.full(E, abi.CHART_ROTATION_ONLY, np.uint8)
        ext[0] = abi.CHART_FULL
        set_charts(w, ext_chart=ext)
    elif kind == "landmarks":
        lm = np.zeros(L, np.uint8)
        lm[::4] = 1
        set_charts(w, lm_fixed=lm)
    return w


KINDS = ["constant", "scoped", "rotation", "landmarks"]


@pytest.mark.parametrize("kind", KINDS)
def test_charted_step_matches_oracle(oracle, backend, kind):
    w = _charted(31, kind)
    nr, L = w.retained_dim(), w.L
    ref = oracle.step(w.window, nr, L, 1e-3)
    assert ref["status"] == 0
    s = backend.Solver()
    s.set_windows([w])
    s.step(1e-3)
    got = s.read_step(0)
    S, rhs = s.read_reduced(0)
    assert got["status"] == 0
    assert rel(S, ref["S"]) < 1e-12
    assert rel(rhs, ref["rhs"]) < 1e-11
    assert rel(got["delta"], ref["delta"]) < 1e-9
    assert np.array_equal(got["delta"] == 0.0, ref["delta"] == 0.0)  # the same increments are exactly zero
    assert abs(got["predicted"] - ref["predicted"]) <= 1e-9 * abs(ref["predicted"])
    assert got["trial_valid"] and abs(got["trial_cost"] - ref["trial_cost"]) <= 1e-10 * abs(ref["trial_cost"])


@pytest.mark.parametrize("kind", ["constant", "rotation"])
def test_charted_step_on_a_wide_window(oracle, backend, kind):
    """The charts on a window of 319 retained columns (18 keyframes, 8 cameras with
    their own extrinsics), which the wide factorization sequence takes (charts
    applied by k_wide_prepare), inside one batch with a narrow window: both
    against the oracle."""
    wide = _charted(33, kind, replace(synth.C3, keyframes=18, landmarks=1500, per_camera_extrinsics=True))
    narrow = _charted(34, kind)
    assert wide.retained_dim() >= 288 > narrow.retained_dim()
    s = backend.Solver()
    s.set_windows([narrow, wide])
    s.step(1e-3)
    for i, w in enumerate([narrow, wide]):
        ref = oracle.step(w.window, w.retained_dim(), w.L, 1e-3)
        got = s.read_step(i)
        S, rhs = s.read_reduced(i)
        assert got["status"] == 0 and ref["status"] == 0
        assert rel(S, ref["S"]) < 1e-12
        assert rel(rhs, ref["rhs"]) < 1e-11
        assert rel(got["delta"], ref["delta"]) < 1e-9
        assert np.array_equal(got["delta"] == 0.0, ref["delta"] == 0.0)
        assert abs(got["predicted"] - ref["predicted"]) <= 1e-9 * abs(ref["predicted"])


@pytest.mark.parametrize("kind", KINDS)
def test_charted_solve_matches_oracle(oracle, backend, kind):
    w = _charted(32, kind)
    x0 = w.state_vector()
    E = w.window.num_extrinsics
    t0 = w.extrinsics().reshape(E, 7)[:, :3].copy()
    st, rep = oracle.lm_solve(w.window, 5)
    assert st == 0
    xo = w.state_vector()
    w.set_state_vector(x0)
    s = backend.Solver()
    s.set_windows([w])
    s.solve(5)
    s.synchronize()
    s.read_states()
    g = s.reports()[0]
    assert g.status == 0 and (g.iterations, g.accepted_steps) == (rep.iterations, rep.accepted_steps)
    assert abs(g.final_cost - rep.final_cost) <= 1e-7 * rep.final_cost
    xg = w.state_vector()
    assert rel(xg - x0, xo - x0) < 1e-6
    assert np.array_equal(xg == x0, xo == x0)  # constant blocks are bit-for-bit untouched on both
    if kind == "rotation":
        assert np.array_equal(w.extrinsics().reshape(E, 7)[1:, :3], t0[1:])


@pytest.mark.parametrize("m", [0, 2, 3])
def test_time_budget_and_minimum_iterations(oracle, backend, m):
    """A budget that has elapsed when the first step is solved (1 ns) stops each window before
    iteration max(min_iterations, 1), as the oracle does with its budget elapsed from the start."""
    ws = [synth.SynthWindow(SPEC, 40 + i) for i in range(3)]
    x0 = [w.state_vector() for w in ws]
    refs = []
    for w in ws:
        st, rep = oracle.lm_solve_options(w.window, 8, min_iterations=m, budget_elapsed=True)
        refs.append((rep, w.state_vector()))
    for w, x in zip(ws, x0):
        w.set_state_vector(x)
    s = backend.Solver(min_iterations=m, time_budget_s=1e-9)
    s.set_windows(ws)
    s.solve(8)
    s.synchronize()
    s.read_states()
    for g, (rep, xo), w, x in zip(s.reports(), refs, ws, x0):
        assert (g.status, g.iterations, g.accepted_steps) == (rep.status, rep.iterations, rep.accepted_steps)
        assert g.iterations == max(m, 1)
        assert rel(w.state_vector() - x, xo - x) < 1e-6 if np.any(xo != x) else np.array_equal(w.state_vector(), x)


def test_long_budget_changes_nothing(backend):
    ws = [synth.SynthWindow(SPEC, 50 + i) for i in range(2)]
    x0 = [w.state_vector() for w in ws]
    out = []
    for opts in (dict(), dict(min_iterations=1, time_budget_s=100.0)):
        for w, x in zip(ws, x0):
            w.set_state_vector(x)
        s = backend.Solver(**opts)
        s.set_windows(ws)
        s.solve(5)
        s.synchronize()
        s.read_states()
        out.append(([(r.iterations, r.accepted_steps) for r in s.reports()], [w.state_vector() for w in ws]))
        s.close()
    assert out[0][0] == out[1][0]
    for a, b in zip(out[0][1], out[1][1]):
        assert rel(a, b) < 1e-9  # the run-to-run order of the FP64 accumulation differs between any two solves


def test_host_factors_match_the_device_prior_and_the_oracle(oracle, backend):
    """Windows 0 and 2 hand their prior over as caller-evaluated factors, window 1 keeps it on the
    device: each result equals the device solve of the window with its own prior, and the oracle's
    solve with the same caller factor."""
    ws = [synth.SynthWindow(SPEC, 60 + i) for i in range(3)]
    x0 = [w.state_vector() for w in ws]
    nr = [w.retained_dim() for w in ws]
    s = backend.Solver()
    s.set_windows(ws)
    s.solve(5)
    s.synchronize()
    s.read_states()
    native = [(r.iterations, r.accepted_steps, r.final_cost) for r in s.reports()]
    xn = [w.state_vector() for w in ws]
    s.close()
    for w, x in zip(ws, x0):
        w.set_state_vector(x)
    bare = [without_prior(ws[0].window), ws[1].window, without_prior(ws[2].window)]
    host = PriorAsHostFactor(oracle, [w.window for w in ws], nr)
    s = backend.Solver()
    s.set_windows(bare)
    s.solve_host(5, host, has_host=[1, 0, 1])
    s.synchronize()
    s.read_states()
    for i, r in enumerate(s.reports()):
        assert r.status == 0 and (r.iterations, r.accepted_steps) == native[i][:2]
        assert abs(r.final_cost - native[i][2]) <= 1e-10 * native[i][2]
        assert rel(ws[i].state_vector() - x0[i], xn[i] - x0[i]) < 1e-8
    assert host.calls[0] >= 2 and host.calls[1] >= 2
    # the oracle with the same caller factor
    ws[0].set_state_vector(x0[0])
    st, rep = oracle.lm_solve_options(without_prior(ws[0].window), 5, host=host, nr=nr[0], window_index=0)
    assert st == 0 and (rep.iterations, rep.accepted_steps) == native[0][:2]


def test_failed_host_evaluation_fails_the_window(backend):
    ws = [synth.SynthWindow(SPEC, 70 + i) for i in range(2)]
    s = backend.Solver()
    s.set_windows(ws)
    s.solve_host(3, lambda w, trial, *a: None, has_host=[1, 0])
    s.synchronize()
    reps = s.reports()
    assert reps[0].status == abi.E_NONFINITE and reps[1].status == 0


def test_solver_device_bytes_grow_only(backend):
    s = backend.Solver()
    s.set_windows([synth.SynthWindow(SPEC, 80)])
    a = s.device_bytes()
    s.set_windows([synth.SynthWindow(replace(SPEC, landmarks=100), 81)])
    assert s.device_bytes() == a > 0


def test_synchronize_and_timing_before_the_first_solve(backend):
    """A caller may synchronize (and read the timing) right after set_windows:
    the timing events were never recorded then, and the next solve (with or
    without per-kernel events) must still launch cleanly."""
    s = backend.Solver()
    s.set_windows([synth.SynthWindow(SPEC, 82)])
    s.synchronize()
    assert s.timing()[0] == 0.0
    s.kernel_times(1)
    s.solve(1)
    s.synchronize()
    kt = s.kernel_times(-1)
    s.kernel_times(0)
    assert kt["linearize"][1] == 1 and kt["factor"][1] >= 1
    assert s.timing()[0] > 0
