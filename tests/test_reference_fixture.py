"""The oracle on the reference's own geometry fixture and tolerances
(src/backend/tests/ManagedWindowRegression.cpp:28-66,119-234; see
reference_fixture.py): analytic Jacobians against central differences in the
left tangent with the reference's steps, the residual against the oracle's
second (numeric-route) residual, exact zeros of same-epoch blocks, and rho = 0
rejected.  The device runs the same cases in test_gpu_reference_fixture.py."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import reference_fixture as RF


def _oracle_factor(O, fw, derivatives=True):
    ok, r, J, flags = O.visual_factor(fw.window, 0, 0, derivatives)
    return ok, r, J


def test_fixture_projects_as_the_reference():
    # camera 0 stops at the point behind it; camera 1 (EUCM) sees all four
    for frame in (1, 2):
        for p in range(3):
            RF.keypoint(frame, 0, p)
        for p in range(4):
            RF.keypoint(frame, 1, p)
    assert RF._pinhole_project(RF.POINTS[3]) is None
    b, _ = RF.observe(1, 1, 3)
    assert b[2] < 0  # full-sphere bearing of the rear anchor


@pytest.mark.parametrize("case", RF.all_cases(), ids=lambda c: f"{c[0]}-s{c[2]}" if isinstance(c, tuple) else str(c))
def test_oracle_matches_reference_numeric_route(oracle, case):
    obs, anchor, scenario = case
    fw = RF.FixtureWindow(obs, anchor, scenario)
    ok, r, J = _oracle_factor(oracle, fw)
    assert ok
    rn = np.zeros(2)
    assert oracle.lib().oracle_visual_residual_numeric(C.byref(fw.window), 0, 0, rn.ctypes.data_as(oracle.dp)) == 1
    assert np.linalg.norm(r - rn) < 1e-8 * (1 + np.linalg.norm(rn))
    rho = fw.arrays["rho"][0]
    for kind, index in fw.blocks():
        width = fw.width(kind)
        numeric = np.zeros((2, width))
        for c in range(width):
            h = fw.step(kind, c, rho)
            okp, rp, _ = _oracle_factor(oracle, fw.perturbed(kind, index, c, h, True), False)
            okm, rm, _ = _oracle_factor(oracle, fw.perturbed(kind, index, c, h, False), False)
            assert okp and okm
            numeric[:, c] = (rp - rm) / (2 * h)
        analytic = fw.analytic_block(J, kind, index)
        tol = 1e-5 if kind in ("extrinsic", "td") else 1e-6
        assert np.linalg.norm(analytic - numeric) <= 1e-7 + tol * np.linalg.norm(numeric), (kind, index)
    if fw.same_epoch:
        assert np.all(J[:, 0:24] == 0.0)  # same-epoch pose and shared extrinsic cancel exactly
    if scenario == 3:
        fw.arrays["rho"][0] = 0.0
        assert not _oracle_factor(oracle, fw, False)[0]


def test_camera_independent_residual_and_fd(oracle):
    """factorGeometryAndJacobians (:119-167): the noise-free temporal EUCM observation has a whitened
    residual below 1e-3 (pixels stored as float), and each tangent column agrees with central
    differences at h = 2e-7 (recordDerivative's default 1e-7 + 1e-6 |numeric|)."""
    fw = RF.FixtureWindow((2, 1, 0), (1, 0, 0), 0)
    ok, r, J = _oracle_factor(oracle, fw)
    assert ok and np.linalg.norm(r) < 1e-3
    h = 2e-7
    for kind, index in fw.blocks():
        for c in range(fw.width(kind)):
            _, rp, _ = _oracle_factor(oracle, fw.perturbed(kind, index, c, h, True), False)
            _, rm, _ = _oracle_factor(oracle, fw.perturbed(kind, index, c, h, False), False)
            numeric = (rp - rm) / (2 * h)
            analytic = fw.analytic_block(J, kind, index)[:, c]
            assert np.linalg.norm(numeric - analytic) <= 1e-7 + 1e-6 * np.linalg.norm(numeric), (kind, index, c)
