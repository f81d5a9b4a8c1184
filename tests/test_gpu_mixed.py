"""Mixed-precision linearization against the FP64 path and the FP64 oracle.

In CGMLI_PRECISION_MIXED the bearing factors' Jacobians and robust weights are
FP32 and the landmark Hessian blocks (d_l and the cross vectors c_l) are summed in
compensated FP32; residuals, costs, gradients, the reduced system, its Cholesky
and the marginalization stay FP64.

Bars:
  * reduced-system step dx      rel 1e-6 against the FP64 oracle (the headline bar) on
                                windows whose gauge is fixed (IMU and a prior, or IMU on
                                the reference's configurations); rel 1e-5 on gauge-free
                                windows, whose free directions only the damping holds
  * full step (with d rho)      the same bars; the depth derivative is formed in FP64
                                (in FP32 it loses its digits for low-parallax observations,
                                and the landmark increments then drift by 1e-5 and more)
  * linearized cost             rel 1e-12 (FP64 residuals: the cost is the FP64 path's)
  * reduced system S            rel 1e-5 (FP32 Jacobian rounding, FP64 sums)
  * LM solve                    the same accepted steps, final cost rel 1e-8, states rel
                                1e-5 of their norm (the reference's GPU-against-Ceres bar
                                is 1e-4, ManagedWindowRegression.cpp:640-691)
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth

pytestmark = pytest.mark.gpu

DX_BAR = 1e-6


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


# windows without a prior whose free directions only the damping holds
GAUGE_FREE = {"no_imu_no_prior", "huber_off"}

SPECS = {
    "tiny": replace(synth.C1, keyframes=4, landmarks=60),
    "c1": synth.C1,
    "c2": synth.C2,
    "shared_calib": replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True,
                            with_prior=True),
    "no_imu_no_prior": replace(synth.C1, keyframes=6, landmarks=300, with_imu=False, outlier_fraction=0.0),
    "huber_off": replace(synth.C1, keyframes=5, landmarks=200, huber=0.0, outlier_fraction=0.0),
    "long_tracks_8cam": replace(synth.C3, keyframes=12, landmarks=1500),
    "c4_draw": synth.c4_spec(np.random.default_rng(11)),
}


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("lam", [1e-4, 1e-2])
def test_mixed_step_within_bar(oracle, backend, name, lam):
    w = synth.SynthWindow(SPECS[name], 17)
    nr, L = w.retained_dim(), w.L
    ref = oracle.step(w.window, nr, L, lam)
    assert ref["status"] == 0
    s = backend.Solver(precision=abi.PRECISION_MIXED)
    s.set_windows([w])
    s.step(lam)
    got = s.read_step(0)
    S, _ = s.read_reduced(0)
    assert got["status"] == 0
    bar = 10 * DX_BAR if name in GAUGE_FREE else DX_BAR
    assert rel(got["delta"][:nr], ref["delta"][:nr]) < bar
    assert rel(got["delta"], ref["delta"]) < bar
    assert abs(got["cost"] - ref["cost"]) <= 1e-12 * abs(ref["cost"])
    assert rel(S, ref["S"]) < 1e-5
    assert got["trial_valid"] and abs(got["trial_cost"] - ref["trial_cost"]) <= 1e-6 * abs(ref["trial_cost"])


def test_mixed_large_window_global_factor_path(oracle, backend):
    """30 keyframes, 8 cameras, track length up to 25: the global-memory Cholesky."""
    w = synth.SynthWindow(replace(synth.C3, landmarks=4000), 3)
    nr, L = w.retained_dim(), w.L
    ref = oracle.step(w.window, nr, L, 1e-4)
    s = backend.Solver(precision=abi.PRECISION_MIXED)
    s.set_windows([w])
    s.step(1e-4)
    got = s.read_step(0)
    assert got["status"] == 0
    assert rel(got["delta"][:nr], ref["delta"][:nr]) < DX_BAR


def test_mixed_batch_step_matches_fp64_path(backend):
    """A batch of windows drawn as the batched configuration: every window's
    mixed step within the bar of the FP64 path's step on the same batch."""
    windows = synth.make_windows("c4", 24, seed=5)
    fp64 = backend.Solver()
    fp64.set_windows(windows)
    fp64.step(1e-4)
    mixed = backend.Solver(precision=abi.PRECISION_MIXED)
    mixed.set_windows(windows)
    mixed.step(1e-4)
    worst, worst_all = 0.0, 0.0
    for i, w in enumerate(windows):
        nr = w.retained_dim()
        a, b = mixed.read_step(i), fp64.read_step(i)
        assert a["status"] == 0 and b["status"] == 0
        worst = max(worst, rel(a["delta"][:nr], b["delta"][:nr]))
        worst_all = max(worst_all, rel(a["delta"], b["delta"]))
        assert a["cost"] == pytest.approx(b["cost"], rel=1e-12)
    assert worst < DX_BAR
    assert worst_all < DX_BAR


def test_mixed_step_same_alone_and_in_batch(backend):
    """The mixed linearization of a window does not depend on its neighbours."""
    windows = synth.make_windows("c4", 6, seed=9)
    batch = backend.Solver(precision=abi.PRECISION_MIXED)
    batch.set_windows(windows)
    batch.step(1e-4)
    for i, w in enumerate(windows):
        alone = backend.Solver(precision=abi.PRECISION_MIXED)
        alone.set_windows([w])
        alone.step(1e-4)
        assert rel(batch.read_step(i)["delta"], alone.read_step(0)["delta"]) < 1e-9


@pytest.mark.parametrize("name,iterations", [("c2", 5), ("long_tracks_8cam", 5)])
def test_mixed_lm_solve_matches_fp64(backend, name, iterations):
    w64 = synth.SynthWindow(SPECS[name], 23)
    wmx = synth.SynthWindow(SPECS[name], 23)
    a = backend.Solver()
    a.set_windows([w64])
    a.solve(iterations)
    a.read_states()
    b = backend.Solver(precision=abi.PRECISION_MIXED)
    b.set_windows([wmx])
    b.solve(iterations)
    b.read_states()
    ra, rb = a.reports()[0], b.reports()[0]
    assert ra.status == rb.status == 0
    assert ra.iterations == rb.iterations and ra.accepted_steps == rb.accepted_steps
    assert rb.final_cost == pytest.approx(ra.final_cost, rel=1e-8)
    assert rel(wmx.state_vector(), w64.state_vector()) < 1e-5


def test_mixed_batched_solve_states(backend):
    windows64 = synth.make_windows("c4", 16, seed=31)
    windowsmx = synth.make_windows("c4", 16, seed=31)
    a = backend.Solver()
    a.set_windows(windows64)
    a.solve(5)
    a.read_states()
    b = backend.Solver(precision=abi.PRECISION_MIXED)
    b.set_windows(windowsmx)
    b.solve(5)
    b.read_states()
    for w64, wmx, ra, rb in zip(windows64, windowsmx, a.reports(), b.reports()):
        assert ra.status == rb.status and ra.accepted_steps == rb.accepted_steps
        assert rb.final_cost == pytest.approx(ra.final_cost, rel=1e-8)
        assert rel(wmx.state_vector(), w64.state_vector()) < 1e-5
