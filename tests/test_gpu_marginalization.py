"""GPU parity of the Schur-complement marginalization prior against the FP64 oracle.

A is unique only up to an orthogonal transform (gauge freedom, rank cutoff), so
the prior is compared through A^T A (information) and A^T r0 (gradient), at
relative 1e-8 (the marginal-prior bar).  The formation scalars (robust cost,
whitened |r|^2, eliminated reduction, cutoff) are compared too; the reference's
known-answer test for them is marginalizationQuadraticAgreement
(tests/test_backend.cpp:235-278), restated on the oracle in test_oracle.py.
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


SPECS = {
    "c1": synth.C1,
    "c2": synth.C2,
    "shared_calib": replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True,
                            with_prior=True),
    "no_imu_no_prior": replace(synth.C1, keyframes=6, landmarks=300, with_imu=False, outlier_fraction=0.0),
    "long_tracks_8cam": replace(synth.C3, keyframes=12, landmarks=1500),
}


def compare(got, ref, tol=1e-8):
    assert got["status"] == 0 and ref["status"] == 0
    assert got["cols"] == ref["cols"]
    assert got["rank"] == ref["rank"]
    assert np.array_equal(got["kinds"], ref["kinds"]) and np.array_equal(got["index"], ref["index"])
    amb = got["reference"].size
    assert np.array_equal(got["reference"], ref["reference"][:amb])
    Ag, Ar = got["A"], ref["A"]
    assert rel(Ag.T @ Ag, Ar.T @ Ar) < tol
    assert rel(Ag.T @ got["r0"], Ar.T @ ref["r0"]) < tol
    for key in ("robust_cost", "rss"):
        assert abs(got[key] - ref[key]) <= 1e-12 * abs(ref[key])
    # the eliminated reduction 1/2 b^T H^+ b is a diagnostic, not part of the
    # prior.  Near an optimum each landmark gradient b_l is a sum of cancelling
    # terms: the device and the oracle evaluate the residuals in different (but
    # equivalent) operation orders, ~1e-13 apart, and the cancellation amplifies
    # that to ~1e-7 in the sum of b_l^2 / d_l
    assert abs(got["eliminated_reduction"] - ref["eliminated_reduction"]) <= 1e-6 * abs(ref["eliminated_reduction"])
    assert abs(got["cutoff"] - ref["cutoff"]) <= tol * ref["cutoff"]


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("policy", [abi.MARGIN_OLD, abi.MARGIN_SECOND_NEW])
def test_prior_matches_oracle(oracle, backend, name, policy):
    w = synth.SynthWindow(SPECS[name], 41)
    victim = 0 if policy == abi.MARGIN_OLD else w.spec.keyframes - 2
    ref = oracle.marginalize_window(w.window, victim, policy)
    s = backend.Solver()
    s.set_windows([w])
    s.marginalize([victim], policy)
    got = s.read_prior(0)
    compare(got, ref)


def test_prior_after_solve_matches_oracle(oracle, backend):
    """Solve then marginalize on the device; the oracle marginalizes the read-back states."""
    w = synth.SynthWindow(SPECS["c2"], 43)
    s = backend.Solver()
    s.set_windows([w])
    s.solve(3)
    s.marginalize([0], abi.MARGIN_OLD)
    got = s.read_prior(0)
    s.read_states()
    ref = oracle.marginalize_window(w.window, 0, abi.MARGIN_OLD)
    compare(got, ref)


def test_batch_marginalization_equals_alone(oracle, backend):
    """Windows of uneven size and different victims/skips in one call."""
    windows = synth.make_windows("c4", 5, seed=91)
    victims = [0, 1, -1, windows[3].spec.keyframes - 2, 0]
    s = backend.Solver()
    s.set_windows(windows)
    s.marginalize(victims, abi.MARGIN_OLD)
    for i, (w, v) in enumerate(zip(windows, victims)):
        got = s.read_prior(i)
        if v < 0:
            assert got["status"] == 0 and got["rank"] == 0 and got["cols"] == 0
            continue
        compare(got, oracle.marginalize_window(w.window, v, abi.MARGIN_OLD))


def test_large_window_second_new(oracle, backend):
    """30 keyframes, 8 cameras, 4000 landmarks: a separator of ~200 columns."""
    w = synth.SynthWindow(replace(synth.C3, landmarks=4000), 5)
    v = w.spec.keyframes - 2
    ref = oracle.marginalize_window(w.window, v, abi.MARGIN_SECOND_NEW)
    s = backend.Solver()
    s.set_windows([w])
    s.marginalize([v], abi.MARGIN_SECOND_NEW)
    compare(s.read_prior(0), ref)


def test_wide_window_landmark_path(oracle, backend):
    """48 keyframes with 32-observation tracks: the eliminated landmarks touch
    about 300 visual columns, above the dense-row path, so the per-landmark
    kernel forms the visual part."""
    w = synth.SynthWindow(replace(synth.C3, keyframes=48, landmarks=3000, track_max=32), 5)
    ref = oracle.marginalize_window(w.window, 0, abi.MARGIN_OLD)
    s = backend.Solver()
    s.set_windows([w])
    s.marginalize([0], abi.MARGIN_OLD)
    compare(s.read_prior(0), ref)


def test_invalid_point_reported(backend):
    """A non-positive inverse distance among the eliminated landmarks makes the
    linearization invalid; the status comes back instead of a prior."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=4, landmarks=60), 8)
    w.rho()[:] = -0.1
    s = backend.Solver()
    s.set_windows([w])
    s.marginalize([0], abi.MARGIN_OLD)
    assert s.read_prior(0)["status"] == 2  # CGMLI_E_NONFINITE


def test_dense_eigen_matches_numpy(backend):
    rng = np.random.default_rng(3)
    for n in (1, 7, 64, 181):
        X = rng.standard_normal((n, max(1, n - 3)))
        H = X @ X.T + np.diag(rng.uniform(0, 1e-3, n))
        ev, U = backend.marg_eigen(H)
        ref = np.linalg.eigvalsh(H)
        assert np.all(np.diff(ev) >= 0)
        assert np.max(np.abs(ev - ref)) <= 1e-12 * np.max(np.abs(ref))
        assert rel(U @ np.diag(ev) @ U.T, H) < 1e-13
        assert np.max(np.abs(U.T @ U - np.eye(n))) < 1e-13


def test_dense_psd_solve_matches_oracle(oracle, backend):
    rng = np.random.default_rng(4)
    n, cols = 40, 9
    X = rng.standard_normal((n, 30))
    H = X @ X.T  # rank 30: the cutoff drops 10 directions
    rhs = rng.standard_normal((n, cols))
    st, ref = oracle.psd_solve(H, rhs, 1e-12, 1e-9)
    assert st == 0
    got = backend.marg_psd_solve(H, rhs)
    assert rel(got, ref) < 1e-10


def test_dense_psd_solve_rejects_indefinite(backend):
    H = np.diag([4.0, 1.0, -1.0])
    with pytest.raises(backend.BackendError) as e:
        backend.marg_psd_solve(H, np.ones(3))
    assert e.value.code == 6  # CGMLI_E_INDEFINITE


def test_dense_subtract(backend):
    rng = np.random.default_rng(5)
    nm, nr = 15, 33
    C = rng.standard_normal((nm, nr))
    Sx = rng.standard_normal((nm, nr + 1))
    H = rng.standard_normal((nr, nr))
    g = rng.standard_normal(nr)
    Ho, go = backend.marg_subtract(C, Sx, H, g)
    full = np.hstack([H, g[:, None]]) - C.T @ Sx
    assert rel(Ho, full[:, :nr]) < 1e-14 and rel(go, full[:, nr]) < 1e-14


def test_diagonal_psd_known_answer_on_device():
    """untouchedPriorAndDiagonalKernel (ManagedWindowRegression.cpp:310-329) through
    cgmli_marg_psd_solve: H = diag(2, 0, 1e-14, 5), rhs = ones(4, 2) gives rows 0.5, 0, 0, 0.2
    within 1e-12; a negative diagonal information must fail."""
    from cgmli_slam_b200 import backend as B

    H = np.diag([2.0, 0.0, 1e-14, 5.0])
    x = B.marg_psd_solve(H, np.ones((4, 2)))
    expected = np.zeros((4, 2))
    expected[0] = 0.5
    expected[3] = 0.2
    assert np.linalg.norm(x - expected) < 1e-12
    H[2, 2] = -1.0
    with pytest.raises(B.BackendError) as e:
        B.marg_psd_solve(H, np.ones((4, 2)))
    assert e.value.code == 6  # CGMLI_E_INDEFINITE
