"""CPU checks of the boundary options on the oracle: solve-time charts, the
time budget with minimum iterations, and caller-evaluated factors
(BackendOptimizer.cpp:44-91,167-307,783-795).  The device is held to the same
results in test_gpu_boundary.py."""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from boundary_cases import PriorAsHostFactor, set_charts, without_prior
from cgmli_slam_b200 import abi, synth

SPEC = replace(synth.C2, landmarks=400)


def test_constant_blocks_select_the_reduced_system(oracle):
    """Constant blocks only remove their rows and columns: the charted system is the full
    damped reduced system restricted to the free columns (identity at the fixed ones)."""
    w = synth.SynthWindow(SPEC, 5)
    nr, L = w.retained_dim(), w.L
    full = oracle.step(w.window, nr, L, 1e-3)
    kf = np.zeros(w.K, np.uint8)
    kf[0] = abi.FIX_POSE | abi.FIX_VELOCITY | abi.FIX_BIAS
    kf[1] = abi.FIX_BIAS
    ext = np.zeros(w.window.num_extrinsics, np.uint8)
    ext[2] = abi.CHART_FIXED
    set_charts(w, kf_fixed=kf, ext_chart=ext)
    got = oracle.step(w.window, nr, L, 1e-3)
    fixed = np.zeros(nr, bool)
    fixed[0:15] = True
    fixed[15 + 9:30] = True
    fixed[15 * w.K + 12:15 * w.K + 18] = True
    free = ~fixed
    assert np.allclose(got["S"][np.ix_(free, free)], full["S"][np.ix_(free, free)], rtol=0, atol=1e-12 * np.abs(full["S"]).max())
    assert np.array_equal(got["S"][np.ix_(fixed, fixed)], np.eye(fixed.sum()))
    assert np.all(got["delta"][:nr][fixed] == 0.0)
    x = np.linalg.solve(full["S"][np.ix_(free, free)], full["rhs"][free])
    assert np.allclose(got["delta"][:nr][free], x, rtol=1e-9, atol=1e-12)


def test_rotation_only_extrinsic_keeps_its_translation(oracle):
    w = synth.SynthWindow(SPEC, 6)
    nr, L = w.retained_dim(), w.L
    E = w.window.num_extrinsics
    ext = np.full(E, abi.CHART_ROTATION_ONLY, np.uint8)
    set_charts(w, ext_chart=ext)
    t0 = w.extrinsics().reshape(E, 7)[:, :3].copy()
    q0 = w.extrinsics().reshape(E, 7)[:, 3:].copy()
    st, rep = oracle.lm_solve(w.window, 5)
    assert st == 0 and rep.accepted_steps > 0
    X = w.extrinsics().reshape(E, 7)
    assert np.array_equal(X[:, :3], t0)  # translation untouched
    assert np.max(np.abs(X[:, 3:] - q0)) > 0  # the rotations moved


def test_rotation_only_system_is_the_restricted_quadratic(oracle):
    """The theta block of a rotation-only extrinsic is M^T S M with M = [[p]x; I], damped by
    lambda max(diag(M^T H M), 1e-6); its right-hand side is M^T rhs."""
    lam = 1e-3
    w = synth.SynthWindow(SPEC, 7)
    nr, L = w.retained_dim(), w.L
    full = oracle.step(w.window, nr, L, lam)
    _, H, *_ = oracle.linearize(w.window, nr, L)
    E = w.window.num_extrinsics
    e = 1
    ext = np.zeros(E, np.uint8)
    ext[e] = abi.CHART_ROTATION_ONLY
    set_charts(w, ext_chart=ext)
    got = oracle.step(w.window, nr, L, lam)
    c0 = 15 * w.K + 6 * e
    p = w.extrinsics().reshape(E, 7)[e, :3]
    P = np.array([[0, -p[2], p[1]], [p[2], 0, -p[0]], [-p[1], p[0], 0]])
    T = np.eye(nr)[:, [i for i in range(nr) if not (c0 <= i < c0 + 3)]]
    T[c0:c0 + 3, np.arange(c0, c0 + 3)] = P  # theta columns stay at c0 + 3 .. c0 + 5 of the reduced index
    Sd = full["S"] - np.diag(lam * np.maximum(np.diag(H), 1e-6))
    Sr = T.T @ Sd @ T + np.diag(lam * np.maximum(np.diag(T.T @ H @ T), 1e-6))
    keep = [i for i in range(nr) if not (c0 <= i < c0 + 3)]
    assert np.allclose(got["S"][np.ix_(keep, keep)], Sr, rtol=0, atol=1e-11 * np.abs(Sr).max())
    assert np.allclose(got["rhs"][keep], T.T @ full["rhs"], rtol=0, atol=1e-11 * np.abs(full["rhs"]).max())
    d = got["delta"][:nr]
    assert np.allclose(d[c0:c0 + 3], P @ d[c0 + 3:c0 + 6], rtol=1e-12, atol=1e-18)


def test_fixed_landmarks_are_not_eliminated(oracle):
    w = synth.SynthWindow(SPEC, 8)
    nr, L = w.retained_dim(), w.L
    lm = np.zeros(L, np.uint8)
    lm[::3] = 1
    set_charts(w, lm_fixed=lm)
    got = oracle.step(w.window, nr, L, 1e-3)
    assert got["status"] == 0 and np.all(got["delta"][nr:][lm == 1] == 0.0)
    assert np.any(got["delta"][nr:][lm == 0] != 0.0)


def test_time_budget_and_minimum_iterations(oracle):
    """An elapsed budget stops before iteration max(min_iterations, 1); without a budget the
    minimum changes nothing."""
    w = synth.SynthWindow(SPEC, 9)
    x0 = w.state_vector()
    st, plain = oracle.lm_solve(w.window, 8)
    assert st == 0 and plain.iterations >= 3
    for m in (0, 1, 2, 3):
        w.set_state_vector(x0)
        st, rep = oracle.lm_solve_options(w.window, 8, min_iterations=m, budget_elapsed=True)
        assert rep.iterations == max(m, 1)
        w.set_state_vector(x0)
        st2, rep2 = oracle.lm_solve_options(w.window, 8, min_iterations=m, budget_elapsed=False)
        assert (rep2.iterations, rep2.accepted_steps) == (plain.iterations, plain.accepted_steps)


def test_host_factor_equals_the_same_factor_on_the_device_path(oracle):
    """The window's prior handed over as a caller-evaluated factor gives the solve of the window
    with its prior."""
    w = synth.SynthWindow(SPEC, 10)
    assert w.window.prior_rank > 0
    x0 = w.state_vector()
    st, ref = oracle.lm_solve(w.window, 5)
    xr = w.state_vector()
    w.set_state_vector(x0)
    bare = without_prior(w.window)
    host = PriorAsHostFactor(oracle, [w.window], [w.retained_dim()])
    st2, rep = oracle.lm_solve_options(bare, 5, host=host, nr=w.retained_dim())
    assert st == st2 == 0
    assert (rep.iterations, rep.accepted_steps) == (ref.iterations, ref.accepted_steps)
    # the host's J^T J is summed in another order than the oracle's own prior accumulation
    assert abs(rep.final_cost - ref.final_cost) <= 1e-10 * ref.final_cost
    assert np.linalg.norm(w.state_vector() - xr) <= 1e-9 * np.linalg.norm(xr - x0)
    assert host.calls[0] >= 1 and host.calls[1] >= 1
