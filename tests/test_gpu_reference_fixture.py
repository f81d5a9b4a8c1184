"""The device on the reference's own geometry fixture and tolerances, through the
C ABI (cgmli_solver_evaluate / cgmli_solver_read_factors, the form of
VisualCudaBatch::evaluate).

analyticSphereDerivativeAgreement (src/backend/tests/ManagedWindowRegression.cpp:
168-234) compares the analytic factor with central differences of the residual
in the left tangent; here both come from the device: the analytic Jacobian of
each case, and the residuals of the same window with one tangent coordinate
moved by +-h (the reference's steps), all windows of all cases solved as one
batch.  Tolerances are the reference's (see reference_fixture.py).  The same
cases run on the oracle in test_reference_fixture.py; the device's Jacobians
are also compared with the oracle's ambient-and-lift route.
"""
from __future__ import annotations

import numpy as np
import pytest

import reference_fixture as RF
from cgmli_slam_b200 import synth

pytestmark = pytest.mark.gpu


def _batch_cases(cases, h_of=None):
    """Base window of every case, then its +-h perturbations; returns the windows and an index."""
    wins, index = [], []
    for case in cases:
        fw = RF.FixtureWindow(*case)
        base = len(wins)
        wins.append(fw)
        pert = {}
        rho = fw.arrays["rho"][0]
        for kind, idx in fw.blocks():
            for c in range(fw.width(kind)):
                h = h_of(kind, c, rho) if h_of else fw.step(kind, c, rho)
                pert[(kind, idx, c)] = (len(wins), len(wins) + 1, h)
                wins.append(fw.perturbed(kind, idx, c, h, True))
                wins.append(fw.perturbed(kind, idx, c, h, False))
        index.append((fw, base, pert))
    return wins, index


def _evaluate(wins, derivatives=True):
    from cgmli_slam_b200 import backend

    s = backend.Solver(device=0)
    s.set_windows([w.window for w in wins])
    s.evaluate(derivatives)
    out = [s.read_factors(i, jacobians=derivatives) for i in range(len(wins))]
    s.close()
    return out


def test_analytic_matches_central_differences_on_device(oracle):
    wins, index = _batch_cases(RF.all_cases())
    res = _evaluate(wins)
    for fw, base, pert in index:
        f = res[base]
        assert f["valid"][0]
        r, J = f["residuals"][0], f["jacobians"][0]
        # the oracle's second residual route (the reference's analytic/numeric residual check)
        rn = np.zeros(2)
        import ctypes as C
        assert oracle.lib().oracle_visual_residual_numeric(C.byref(fw.window), 0, 0, rn.ctypes.data_as(oracle.dp)) == 1
        assert np.linalg.norm(r - rn) < 1e-8 * (1 + np.linalg.norm(rn))
        # and the oracle's analytic factor (ambient Jacobian lifted by the PlusJacobian)
        ok, ro, Jo, _ = oracle.visual_factor(fw.window, 0, 0, True)
        assert ok
        assert np.max(np.abs(r - ro)) <= 1e-13 * (1 + np.max(np.abs(ro)))
        assert np.max(np.abs(J - Jo)) <= 1e-11 * np.max(np.abs(Jo))
        for kind, idx in fw.blocks():
            width = fw.width(kind)
            numeric = np.zeros((2, width))
            for c in range(width):
                ip, im, h = pert[(kind, idx, c)]
                assert res[ip]["valid"][0] and res[im]["valid"][0]
                numeric[:, c] = (res[ip]["residuals"][0] - res[im]["residuals"][0]) / (2 * h)
            analytic = fw.analytic_block(J, kind, idx)
            tol = 1e-5 if kind in ("extrinsic", "td") else 1e-6
            assert np.linalg.norm(analytic - numeric) <= 1e-7 + tol * np.linalg.norm(numeric), (kind, idx)
        if fw.same_epoch:
            assert np.all(J[:, 0:24] == 0.0)  # same-epoch pose and shared extrinsic cancel exactly


def test_residual_only_path_and_invalid_inverse_distance():
    """The residual-only evaluation equals the residual of the full one (the reference's
    residual-only fast path, 1e-11), and rho = 0 is rejected (scenario 3)."""
    cases = RF.all_cases()
    wins = [RF.FixtureWindow(*c) for c in cases]
    full, short = _evaluate(wins, True), _evaluate(wins, False)
    for a, b in zip(full, short):
        assert np.linalg.norm(a["residuals"] - b["residuals"]) <= 1e-11
    bad = [RF.FixtureWindow(o, a, 3, rho_scale=0.0) for o, a, s in cases if s == 3]
    for f in _evaluate(bad, False):
        assert not f["valid"][0]


def test_camera_independent_residual_on_device():
    """factorGeometryAndJacobians (:119-167) on the device: |r| < 1e-3 for the noise-free temporal
    EUCM observation, each column within 1e-7 + 1e-6 |numeric| of central differences at h = 2e-7."""
    wins, index = _batch_cases([((2, 1, 0), (1, 0, 0), 0)], h_of=lambda kind, c, rho: 2e-7)
    res = _evaluate(wins)
    fw, base, pert = index[0]
    J = res[base]["jacobians"][0]
    assert np.linalg.norm(res[base]["residuals"][0]) < 1e-3
    for kind, idx in fw.blocks():
        for c in range(fw.width(kind)):
            ip, im, h = pert[(kind, idx, c)]
            numeric = (res[ip]["residuals"][0] - res[im]["residuals"][0]) / (2 * h)
            analytic = fw.analytic_block(J, kind, idx)[:, c]
            assert np.linalg.norm(numeric - analytic) <= 1e-7 + 1e-6 * np.linalg.norm(numeric), (kind, idx, c)


def test_evaluate_matches_oracle_on_generated_windows(oracle):
    """Every factor of configuration-2 windows (moving bearings, per-camera extrinsics, td) and a
    shared-extrinsic window: residuals, validity and tangent Jacobians against the oracle."""
    from dataclasses import replace

    specs = [replace(synth.C2, landmarks=300), replace(synth.C1, landmarks=200, estimate_extrinsics=True, estimate_td=True,
                                                        with_velocity=True)]
    ws = [synth.SynthWindow(sp, 40 + i) for i, sp in enumerate(specs)]
    res = _evaluate_synth(ws)
    for w, f in zip(ws, res):
        win = w.window
        begin = np.ctypeslib.as_array(win.lm_obs_begin, shape=(w.L + 1,))
        for l in range(w.L):
            for k in range(begin[l], begin[l + 1]):
                ok, r, J, _ = oracle.visual_factor(win, l, k, True)
                assert bool(ok) == bool(f["valid"][k])
                if not ok:
                    continue
                assert np.max(np.abs(f["residuals"][k] - r)) <= 1e-12 * (1 + np.max(np.abs(r)))
                assert np.max(np.abs(f["jacobians"][k] - J)) <= 1e-10 * (1 + np.max(np.abs(J)))


def _evaluate_synth(ws):
    from cgmli_slam_b200 import backend

    s = backend.Solver(device=0)
    s.set_windows(ws)
    s.evaluate(True)
    out = [s.read_factors(i) for i in range(len(ws))]
    s.close()
    return out


def _audit_rel(a, b):
    """relative() of VisualBatchAudit.cpp:23-25: |a - b| / max(1, |a|)."""
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(1.0, np.linalg.norm(a)))


@pytest.mark.parametrize("name", ["c1", "c2"])
def test_reference_audit_bars(oracle, name):
    """The reference's runtime audit (VisualBatchAudit.cpp:24-113), device against the oracle on the
    configuration-1 and -2 windows: stacked residuals and Jacobians within 1e-8, cost within
    1e-8 max(1, |cost|), and the step of the reduced system damped by 1e-3 max(H_ii, 1e-6) (landmarks
    included) within 1e-6."""
    from cgmli_slam_b200 import backend

    w = synth.make_windows(name, 1, seed=88)[0]
    nr, L = w.retained_dim(), w.L
    s = backend.Solver(device=0)
    s.set_windows([w])
    s.evaluate(True)
    f = s.read_factors(0)
    s.step(1e-3)
    step = s.read_step(0)
    s.close()
    win = w.window
    begin = np.ctypeslib.as_array(win.lm_obs_begin, shape=(L + 1,))
    r_ref, J_ref = np.zeros((w.F, 2)), np.zeros((w.F, 2, 26))
    for l in range(L):
        for k in range(begin[l], begin[l + 1]):
            ok, r_ref[k], J_ref[k], _ = oracle.visual_factor(win, l, k, True)
    assert _audit_rel(r_ref.ravel(), f["residuals"].ravel()) < 1e-8
    assert _audit_rel(J_ref.ravel(), f["jacobians"].ravel()) < 1e-8
    ref = oracle.step(win, nr, L, 1e-3)
    assert abs(step["cost"] - ref["cost"]) < 1e-8 * max(1.0, abs(ref["cost"]))
    assert _audit_rel(ref["delta"], step["delta"]) < 1e-6
