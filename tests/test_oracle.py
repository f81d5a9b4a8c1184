"""CPU tests of the FP64 oracle against the reference's own known answers,
fixtures and derivative checks (src/backend/tests/ManagedWindowRegression.cpp,
src/pipeline/tests/NativeSlamRegression.cpp)."""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import replace
from pathlib import Path

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth

GOLDEN = Path(__file__).resolve().parent / "golden"


def _p(a):
    return a.ctypes.data_as(abi.c_double_p)


# ---------------------------------------------------------------- known answers
def test_marginalization_quadratic_agreement(oracle):
    """marginalizationQuadraticAgreement (ManagedWindowRegression.cpp:235-278)."""
    x = np.array([0.3, -0.4])  # eliminated m, retained r
    J = np.array([[2.0, 1.0], [1.0, 3.0]])

    def residual(v):
        return np.array([2 * v[0] + v[1] - 3, v[0] + 3 * v[1] + 1])

    r = residual(x)
    H, g, cost, rss = oracle.robust_normal(J, r, 0.0)
    assert abs(rss - 7.85) < 1e-10
    assert abs(cost - 3.925) < 1e-10
    out = oracle.marginalize_system(H, g, [(1, 1, 0), (1, 0, 0)])
    assert out["status"] == 0 and out["rank"] == 1 and out["nr"] == 1
    A, b = out["A"], out["r0"]
    assert abs((A.T @ A)[0, 0] - 5) < 1e-10
    assert abs((A.T @ b)[0] - 3) < 1e-10
    assert abs(out["eliminated_reduction"] - 3.025) < 1e-10
    offset = 0.5 * rss - out["eliminated_reduction"] - 0.5 * out["new_reference_norm"] ** 2
    assert abs(offset) < 1e-10
    base = 0.9
    for delta in (-1.0, -0.1, 0.0, 0.1, 1.0):
        full = residual(np.array([1.4 - delta, -0.4 + delta]))
        prior = b + A @ np.array([delta])
        err = abs((0.5 * full @ full - base) - (0.5 * prior @ prior - 0.5 * b @ b))
        assert err < 1e-10


def test_diagonal_psd_solve(oracle):
    """untouchedPriorAndDiagonalKernel (ManagedWindowRegression.cpp:310-329)."""
    H = np.diag([2.0, 0.0, 1e-14, 5.0])
    st, x = oracle.psd_solve(H, np.ones((4, 2)))
    expected = np.zeros((4, 2))
    expected[0] = 0.5
    expected[3] = 0.2
    assert st == 0 and np.linalg.norm(x - expected) < 1e-12
    H[2, 2] = -1.0
    st, _ = oracle.psd_solve(H, np.ones((4, 2)))
    assert st == 6  # CGMLI_E_INDEFINITE


def test_general_psd_solve_matches_numpy(oracle):
    rng = np.random.default_rng(3)
    B = rng.normal(size=(6, 4))
    H = B @ B.T  # rank 4
    rhs = rng.normal(size=(6, 3))
    st, x = oracle.psd_solve(H, rhs)
    w, U = np.linalg.eigh(H)
    cut = max(1e-12, 1e-9 * w.max())
    expected = U @ np.diag(np.where(w > cut, 1 / np.where(w > cut, w, 1), 0)) @ U.T @ rhs
    assert st == 0 and np.allclose(x, expected, rtol=1e-10, atol=1e-12)


def test_robust_normal_equations_384x8_golden(oracle):
    """parallelNormalEquationsPreservePrior fixture (ManagedWindowRegression.cpp:279-309)."""
    gold = np.load(GOLDEN / "normal_384x8.npz")
    H, g, cost, _ = oracle.robust_normal(gold["J"], gold["r"], 1.0)
    assert np.linalg.norm(H - gold["H"]) < 1e-9
    assert np.linalg.norm(g - gold["g"]) < 1e-10
    assert abs(cost - float(gold["robust_cost"])) < 1e-12
    out = oracle.marginalize_system(H, g, [(4, 1, 0), (4, 0, 0)])
    A, r0 = out["A"], out["r0"]
    assert np.linalg.norm(A.T @ A - gold["H_prior"]) < 1e-9
    assert np.linalg.norm(A.T @ r0 - gold["b_prior"]) < 1e-10


def test_golden_fixture_is_reproducible(tmp_path):
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", GOLDEN / "make_golden.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.HERE = tmp_path
    mod.normal_384x8()
    a, b = np.load(tmp_path / "normal_384x8.npz"), np.load(GOLDEN / "normal_384x8.npz")
    for k in b.files:
        assert np.array_equal(a[k], b[k]), k


def test_eigen_sym_matches_numpy(oracle):
    rng = np.random.default_rng(1)
    B = rng.normal(size=(30, 30))
    H = B + B.T
    st, ev, V = oracle.eigen_sym(H)
    assert st == 0
    assert np.allclose(ev, np.linalg.eigvalsh(H), rtol=1e-12, atol=1e-12)
    assert np.allclose(V @ np.diag(ev) @ V.T, H, atol=1e-11)


# ---------------------------------------------------------------- derivative checks
SMALL = replace(synth.C1, keyframes=4, landmarks=40, estimate_extrinsics=True, estimate_td=True, with_velocity=True)
SPLIT = replace(SMALL, per_camera_extrinsics=True)


def _lm_ranges(w):
    return np.ctypeslib.as_array(w.window.lm_obs_begin, shape=(w.L + 1,))


def _perturbed(w, block, column, h, l, f):
    """Returns residual of factor f after a left-tangent perturbation h of one block."""
    O = __import__("oracle")
    W = w.window
    a = W.lm_anchor_kf[l]
    b = W.obs_kf[f]
    ea = W.cam_ext[W.lm_anchor_cam[l]]
    eb = W.cam_ext[W.obs_cam[f]]
    restore = None
    if block in ("anchor", "observer", "ext_a", "ext_b"):
        arr = w.poses() if block in ("anchor", "observer") else w.extrinsics()
        idx = {"anchor": a, "observer": b, "ext_a": ea, "ext_b": eb}[block]
        x = arr[7 * idx:7 * idx + 7].copy()
        d = np.zeros(6)
        d[column] = h
        y = np.zeros(7)
        O.lib().oracle_pose_plus(_p(x), _p(d), _p(y))
        arr[7 * idx:7 * idx + 7] = y
        restore = (arr, slice(7 * idx, 7 * idx + 7), x)
    elif block == "td":
        arr = w.td()
        restore = (arr, slice(0, 1), arr[:1].copy())
        arr[0] += h
    else:
        arr = w.rho()
        restore = (arr, slice(l, l + 1), arr[l:l + 1].copy())
        arr[l] += h
    ok, r, _, _ = O.visual_factor(w.window, l, f, derivatives=False)
    restore[0][restore[1]] = restore[2]
    return ok, r


@pytest.mark.parametrize("spec", [SMALL, SPLIT], ids=["shared_extrinsic", "per_camera_extrinsic"])
def test_sphere_jacobians_match_central_differences(oracle, spec):
    """factorGeometryAndJacobians (ManagedWindowRegression.cpp:119-167): analytic
    left-tangent Jacobian vs central differences, h = 2e-7."""
    w = synth.SynthWindow(spec, 11)
    rng = _lm_ranges(w)
    h = 2e-7
    checked = 0
    for l in range(0, w.L, 3):
        for f in range(rng[l], rng[l + 1]):
            ok, r, J, flags = oracle.visual_factor(w.window, l, f)
            assert ok
            blocks = [("anchor", 0, 6), ("observer", 6, 6), ("ext_a", 12, 6), ("td", 24, 1), ("rho", 25, 1)]
            if flags[1]:
                blocks.append(("ext_b", 18, 6))
            for name, off, n in blocks:
                if name in ("anchor", "observer") and flags[0]:
                    assert np.all(J[:, off:off + 6] == 0.0), "same-epoch pose columns must be exactly zero"
                    continue
                for c in range(n):
                    okp, rp = _perturbed(w, name, c, h, l, f)
                    okm, rm = _perturbed(w, name, c, -h, l, f)
                    assert okp and okm
                    numeric = (rp - rm) / (2 * h)
                    analytic = J[:, off + c]
                    scale = max(np.linalg.norm(numeric), 1e-3)
                    assert np.linalg.norm(numeric - analytic) / scale < 2e-5, (name, c)
            checked += 1
    assert checked > 10


def test_analytic_matches_numeric_residual(oracle):
    """analyticSphereDerivativeAgreement (ManagedWindowRegression.cpp:168-234): the
    analytic factor's residual agrees with the numeric reference residual
    (explicit camera chain, FromTwoVectors transport) within 1e-8 (1 + |r|)."""
    for spec in (replace(SMALL, with_velocity=False), SMALL, SPLIT):
        w = synth.SynthWindow(spec, 5)
        w.td()[0] = 0.004
        rng = _lm_ranges(w)
        for l in range(w.L):
            for f in range(rng[l], rng[l + 1]):
                ok, r, _, _ = oracle.visual_factor(w.window, l, f)
                rn = np.zeros(2)
                okn = oracle.lib().oracle_visual_residual_numeric(C.byref(w.window), l, f, _p(rn))
                assert ok and okn
                assert np.linalg.norm(r - rn) < 1e-8 * (1 + np.linalg.norm(rn))


def test_invalid_inverse_depth_rejected(oracle):
    w = synth.SynthWindow(SMALL, 2)
    w.rho()[0] = 0.0
    ok, *_ = oracle.visual_factor(w.window, 0, 0)
    assert not ok
    w.rho()[0] = float("nan")
    ok, *_ = oracle.visual_factor(w.window, 0, 0)
    assert not ok


def test_imu_jacobian_matches_central_differences(oracle):
    """bodyImuJacobianAndFrozenCost (NativeSlamRegression.cpp:601-650): per-block FD."""
    w = synth.SynthWindow(replace(SMALL, landmarks=10), 4)
    W = w.window
    P, S = w.poses(), w.speed_bias()
    for i in range(W.num_imu):
        k = W.imu_kf[i]
        x = [P[7 * k:7 * k + 7].copy(), S[9 * k:9 * k + 9].copy(), P[7 * k + 7:7 * k + 14].copy(), S[9 * k + 9:9 * k + 18].copy()]
        r = np.zeros(15)
        J = np.zeros((15, 30))

        def ev(xs):
            rr = np.zeros(15)
            assert oracle.lib().oracle_imu_factor(C.byref(W.imu[i]), _p(xs[0]), _p(xs[1]), _p(xs[2]), _p(xs[3]), _p(rr), None)
            return rr

        assert oracle.lib().oracle_imu_factor(C.byref(W.imu[i]), _p(x[0]), _p(x[1]), _p(x[2]), _p(x[3]), _p(r), _p(J))
        col0 = [0, 6, 15, 21]
        for b, width in enumerate([6, 9, 6, 9]):
            for c in range(width):
                num = []
                for sgn in (1, -1):
                    xs = [v.copy() for v in x]
                    h = 1e-6
                    if b % 2 == 0:
                        d = np.zeros(6)
                        d[c] = sgn * h
                        y = np.zeros(7)
                        oracle.lib().oracle_pose_plus(_p(x[b]), _p(d), _p(y))
                        xs[b] = y
                    else:
                        xs[b][c] += sgn * h
                    num.append(ev(xs))
                numeric = (num[0] - num[1]) / (2e-6)
                analytic = J[:, col0[b] + c]
                assert np.linalg.norm(numeric - analytic) <= 1e-5 * max(1.0, np.linalg.norm(analytic)), (i, b, c)


def test_prior_chart_derivative_analytic_vs_reference_fd(oracle):
    """The analytic inverse SE(3) left Jacobian equals the reference's
    central-difference chart derivative (VisualCudaBatch.cu:234-245) to FD accuracy."""
    rng = np.random.default_rng(9)
    for _ in range(20):
        x = np.zeros(7)
        ref = np.zeros(7)
        d = np.concatenate([rng.normal(scale=0.3, size=3), rng.normal(scale=0.2, size=3)])
        ref[3:] = [0, 0, 0, 1]
        ref[:3] = rng.normal(size=3)
        oracle.lib().oracle_pose_plus(_p(ref), _p(d), _p(x))
        Da, Df = np.zeros(36), np.zeros(36)
        oracle.lib().oracle_chart_derivative(_p(x), _p(ref), 0, _p(Da))
        oracle.lib().oracle_chart_derivative(_p(x), _p(ref), 1, _p(Df))
        assert np.linalg.norm(Da - Df) < 1e-7 * max(1, np.linalg.norm(Df))


def test_lm_follows_reference_rules(oracle):
    """One resident LM iteration: gain ratio, acceptance and lambda update of
    solveVisualSchur (BackendOptimizer.cpp:246-306)."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=120), 21)
    nr, L = w.retained_dim(), w.L
    x0 = w.state_vector()
    st = oracle.step(w.window, nr, L, 1e-4)
    assert st["status"] == 0
    gain = (st["cost"] - st["trial_cost"]) / st["predicted"]
    status, rep = oracle.lm_solve(w.window, 1)
    assert status == 0 and rep.accepted_steps == 1 and rep.iterations == 1
    lam = max(1e-12, 1e-4 * max(1 / 3, 1 - (2 * gain - 1) ** 3))
    assert math.isclose(rep.lambda_, lam, rel_tol=1e-12)
    assert math.isclose(rep.final_cost, st["trial_cost"], rel_tol=1e-12)
    w.set_state_vector(x0)
    status, rep5 = oracle.lm_solve(w.window, 6)
    assert status == 0 and rep5.final_cost < rep.final_cost


def test_window_marginalization_prior_properties(oracle):
    """Schur prior of an OLD marginalization: PSD, A^T A reproduces the kept
    eigenspace of the Schur information, A^T r0 its gradient."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=150, estimate_extrinsics=True, estimate_td=True,
                                  with_velocity=True, with_prior=True), 8)
    out = oracle.marginalize_window(w.window, 0, abi.MARGIN_OLD)
    assert out["status"] == 0
    H, b, A, r0 = out["H"], out["b"], out["A"], out["r0"]
    wv, U = np.linalg.eigh(H)
    assert wv.min() > -10 * out["cutoff"]
    keep = wv > out["cutoff"]
    Hk = U[:, keep] @ np.diag(wv[keep]) @ U[:, keep].T
    assert np.linalg.norm(A.T @ A - Hk) <= 1e-9 * np.linalg.norm(H)
    assert np.linalg.norm(A.T @ r0 - U[:, keep] @ U[:, keep].T @ b) <= 1e-9 * max(1.0, np.linalg.norm(b))
    # the victim (keyframe 0) is not a separator block
    assert not any(k in (abi.PRIOR_POSE, abi.PRIOR_SPEED_BIAS) and i == 0 for k, i in zip(out["kinds"], out["index"]))
