"""CPU tests of the oracle's conditional calibration information
(BackendOptimizer::calibrationInformation, src/backend/BackendOptimizer.cpp:1084-1170)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from cgmli_slam_b200 import abi, synth

SHARED = replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True, with_prior=True)


def test_layout_and_definiteness(oracle):
    """One block per extrinsic ([theta, p], 6) then the time offset (1); the
    matrix is symmetric positive semidefinite with the reported spectrum."""
    for spec, nblk in ((synth.C1, 1), (synth.C2, 4)):
        w = synth.SynthWindow(spec, 81)
        r = oracle.calibration_information(w.window)
        assert r["status"] == 0
        assert list(r["kinds"]) == [abi.PRIOR_EXTRINSIC] * nblk + [abi.PRIOR_TIME_OFFSET]
        C, ev = r["conditional"], r["eigenvalues"]
        assert C.shape == (6 * nblk + 1,) * 2 and np.array_equal(C, C.T)
        assert np.all(ev >= 0) and np.all(np.diff(ev) >= 0)
        assert np.allclose(np.linalg.eigvalsh(C), ev, rtol=0, atol=1e-9 * ev.max())


def test_prior_adds_information(oracle):
    """A Schur complement is monotone: including the historical prior (a PSD
    term) can only add conditional calibration information."""
    w = synth.SynthWindow(SHARED, 82)
    a = oracle.calibration_information(w.window, False)
    b = oracle.calibration_information(w.window, True)
    assert a["status"] == 0 and b["status"] == 0
    d = np.linalg.eigvalsh(b["conditional"] - a["conditional"])
    assert d.min() >= -1e-8 * np.abs(b["eigenvalues"]).max()
    assert d.max() > 0


def test_visual_information_raises_the_conditional(oracle):
    """Scaling every visual whitening row by 3 scales the visual information by 9
    while the IMU factors and the prior stay: the conditional calibration
    information grows."""
    w = synth.SynthWindow(SHARED, 83)
    r = oracle.calibration_information(w.window, True)
    assert r["status"] == 0
    P = np.ctypeslib.as_array(w.window.obs_P, shape=(6 * w.F,)).copy()
    scaled = np.ascontiguousarray(3.0 * P)
    win = abi.Window.from_buffer_copy(w.window)
    win.obs_P = scaled.ctypes.data_as(abi.c_double_p)
    s = oracle.calibration_information(win, True)
    assert s["status"] == 0
    assert np.trace(s["conditional"]) > np.trace(r["conditional"])


def test_window_without_visual_factors_is_rejected(oracle):
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=0, with_prior=False), 84)
    r = oracle.calibration_information(w.window)
    assert r["status"] == abi.E_INVALID  # no calibration Jacobians
