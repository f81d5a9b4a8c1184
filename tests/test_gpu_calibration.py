"""GPU parity of the conditional calibration information
(cgmli_solver_calibration_information) with the FP64 oracle's restatement of
BackendOptimizer::calibrationInformation (src/backend/BackendOptimizer.cpp:
1084-1170): the conditional and its eigenvalues at relative 1e-8 of their norm
(the marginal-prior bar; measured up to 1.1e-9, the nuisance block's
pseudo-inverse carrying most of it), the same blocks, a symmetric matrix and
non-negative ascending eigenvalues."""
from __future__ import annotations

from dataclasses import replace

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


SPECS = {
    "c1": synth.C1,
    "c2": synth.C2,
    "shared_calib": replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True,
                            with_prior=True),
    "long_tracks_8cam": replace(synth.C3, keyframes=12, landmarks=1500),
}


def compare(got, ref):
    assert got["status"] == 0 and ref["status"] == 0
    assert np.array_equal(got["kinds"], ref["kinds"]) and np.array_equal(got["index"], ref["index"])
    assert rel(got["conditional"], ref["conditional"]) < 1e-8
    assert rel(got["eigenvalues"], ref["eigenvalues"]) < 1e-8
    assert np.all(np.diff(got["eigenvalues"]) >= 0) and np.all(got["eigenvalues"] >= 0)
    C = got["conditional"]
    assert np.array_equal(C, C.T)


@pytest.mark.parametrize("name", list(SPECS))
@pytest.mark.parametrize("prior", [False, True])
def test_calibration_information_matches_oracle(oracle, backend, name, prior):
    w = synth.SynthWindow(SPECS[name], 81)
    ref = oracle.calibration_information(w.window, prior)
    s = backend.Solver()
    s.set_windows([w])
    s.calibration_information(include_prior=prior)
    compare(s.read_calibration_information(0), ref)


def test_visual_only_window_is_indefinite(oracle, backend):
    """Without IMU factors the poses keep a scale gauge that the extrinsic
    translation couples to: the coupling leaves the nuisance block's range, the
    conditional is indefinite, and both report CGMLI_E_INDEFINITE."""
    w = synth.SynthWindow(replace(synth.C1, keyframes=6, landmarks=300, with_imu=False, outlier_fraction=0.0), 81)
    ref = oracle.calibration_information(w.window, False)
    assert ref["status"] == 6  # CGMLI_E_INDEFINITE
    s = backend.Solver()
    s.set_windows([w])
    s.calibration_information(include_prior=False)
    assert s.read_calibration_information(0)["status"] == ref["status"]


def test_batch_after_solve(oracle, backend):
    """Solved windows of the batched workload, evaluated together; each as the
    oracle on the read-back states."""
    windows = synth.make_windows("c4", 4, seed=83)
    s = backend.Solver()
    s.set_windows(windows)
    s.solve(3)
    s.calibration_information(include_prior=True)
    got = [s.read_calibration_information(i) for i in range(len(windows))]
    s.read_states()
    for w, g in zip(windows, got):
        compare(g, oracle.calibration_information(w.window, True))
    # the formation buffers now hold the calibration result, not a prior
    assert s.read_prior(0)["status"] == abi.E_INVALID
