"""GPU parity of the batched IMU preintegration (cgmli_imu_preintegrate) with
the FP64 oracle's restatement of ImuError::redoPreintegration
(src/factor/ImuError.cpp:254-462).

Bars: deltas, bias Jacobians and gyro readings rel 1e-12 (same recursion,
rounding order differs); the whitening through W^T W = P^-1 rel 1e-10 (W is
unique only up to the eigenvector signs and the order within equal
eigenvalues); the device W must invert the oracle's covariance to 1e-10."""
from __future__ import annotations

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


FIELDS = ["delta_quaternion", "delta_velocity", "delta_position", "rotation_gyro", "velocity_gyro", "position_gyro",
          "velocity_accel", "position_accel", "gyros"]


def compare(got, ref, cov):
    assert got.duration == ref.duration and got.gravity == ref.gravity
    assert list(got.reference_bias) == list(ref.reference_bias)
    assert list(got.sensor_position) == list(ref.sensor_position)
    assert list(got.sensor_quaternion) == list(ref.sensor_quaternion)
    for name in FIELDS:
        assert rel(getattr(got, name), getattr(ref, name)) < 1e-12, name
    Wg = np.array(got.whitening).reshape(15, 15, order="F")
    Wr = np.array(ref.whitening).reshape(15, 15, order="F")
    assert rel(Wg.T @ Wg, Wr.T @ Wr) < 1e-10
    assert np.abs(Wg @ cov @ Wg.T - np.eye(15)).max() < 1e-10
    # ascending eigenvalues: row norms of W descend
    n = np.linalg.norm(Wg, axis=1)
    assert np.all(np.diff(n) <= 1e-10 * n[0])


def run_both(oracle, backend, s, prm=None):
    prm = prm or synth.imu_parameters()
    st, ref, cov = oracle.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias, covariance=True)
    assert st == 0
    got = backend.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    return got, ref, cov


@pytest.mark.parametrize("on_sample", [False, True])
def test_batch_matches_oracle(oracle, backend, on_sample):
    """64 rigs x 10 keyframes: 576 intervals with overlapping sample ranges."""
    s = synth.imu_stream(64, 10, 21, on_sample=on_sample)
    got, ref, cov = run_both(oracle, backend, s)
    for i in range(s.count):
        compare(got[i], ref[i], cov[i])


def test_long_interval_many_chunks(oracle, backend):
    """1 kHz samples over 2.1 s: ~2100 steps (66 chunks of 32) per interval."""
    s = synth.imu_stream(3, 2, 22, rate=1000.0, spacing_s=2.1)
    got, ref, cov = run_both(oracle, backend, s)
    for i in range(s.count):
        compare(got[i], ref[i], cov[i])


def test_interval_inside_one_sample_pair(oracle, backend):
    """t0 and t1 between the same two samples: one step, interpolated at both ends."""
    s = synth.imu_stream(1, 2, 23)
    b = s.ranges[0][0] + 3
    t0 = s.time_ns[b] + 1_000_000
    s.t0_ns[0], s.t1_ns[0] = t0, t0 + 2_500_000
    s.ranges[0] = (b, b + 2)
    got, ref, cov = run_both(oracle, backend, s)
    compare(got[0], ref[0], cov[0])


def test_saturated_readings(oracle, backend):
    s = synth.imu_stream(4, 4, 24)
    s.readings[10::17, 1] = 9.0     # gyro above 7.8 rad/s
    s.readings[5::23, 4] = -180.0   # accelerometer above 176 m/s^2
    got, ref, cov = run_both(oracle, backend, s)
    for i in range(s.count):
        compare(got[i], ref[i], cov[i])


def test_stationary_known_answer(oracle, backend):
    n = 201
    t = (np.arange(n, dtype=np.int64) * 1_000_000_000) // 200
    rd = np.tile([0.0, 0.0, 0.0, 0.0, 0.0, 9.81], (n, 1))
    prm = synth.imu_parameters(sigma_g_c=0.002, sigma_a_c=0.02, sigma_gw_c=0.0002, sigma_aw_c=0.002, g_max=100, a_max=100)
    got = backend.imu_preintegrate(prm, t, rd, [[0, n]], [500_000_000], [550_000_000], np.zeros((1, 6)))[0]
    assert list(got.delta_quaternion) == [0.0, 0.0, 0.0, 1.0]
    assert np.allclose(got.delta_velocity, [0, 0, 0.05 * 9.81], rtol=1e-14, atol=1e-15)
    assert np.allclose(np.array(got.rotation_gyro).reshape(3, 3), 0.05 * np.eye(3), rtol=0, atol=1e-15)


def test_invalid_interval_reported(backend):
    s = synth.imu_stream(2, 4, 25)
    prm = synth.imu_parameters()
    t = s.time_ns.copy()
    b = s.ranges[4][0]
    t[b + 6] = t[b + 5]  # repeated time stamp inside interval 4's range
    with pytest.raises(backend.BackendError) as e:
        backend.imu_preintegrate(prm, t, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    assert e.value.code == abi.E_INVALID
    assert "interval" in str(e.value)
    bad = s.ranges.copy()
    bad[2] = (bad[2][0], len(s.time_ns) + 1)  # past the samples: rejected on the host
    with pytest.raises(backend.BackendError) as e:
        backend.imu_preintegrate(prm, s.time_ns, s.readings, bad, s.t0_ns, s.t1_ns, s.bias)
    assert e.value.code == abi.E_INVALID
    # the workspace stays usable
    got = backend.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    assert np.isfinite(np.array(got[0].whitening)).all()


def test_preintegrated_factor_solves_like_oracle(oracle, backend):
    """A device-preintegrated factor placed in a window gives the same LM step on
    the device as on the oracle."""
    from dataclasses import replace
    w = synth.SynthWindow(replace(synth.C1, keyframes=5, landmarks=200), 31)
    K = w.spec.keyframes
    s = synth.imu_stream(1, K, 32, spacing_s=0.3)
    got = backend.imu_preintegrate(synth.imu_parameters(), s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    assert w.window.num_imu == K - 1
    for i in range(K - 1):
        w.window.imu[i] = got[i]
    nr, L = w.retained_dim(), w.L
    ref = oracle.step(w.window, nr, L, 1e-4)
    assert ref["status"] == 0
    sv = backend.Solver()
    sv.set_windows([w])
    sv.step(1e-4)
    g = sv.read_step(0)
    assert g["status"] == 0 and rel(g["delta"], ref["delta"]) < 1e-9


def test_resident_refresh_replaces_drifted_factors(oracle, backend):
    """set_imu_samples + refresh_imu: factors whose first keyframe's bias moved
    past 3e-4 (gyro) or 0.02 (accelerometer) are re-preintegrated on the device at
    the current bias; the others stay bit-identical; the next step uses them."""
    from dataclasses import replace
    w = synth.SynthWindow(replace(synth.C1, keyframes=6, landmarks=200), 33)
    K, nimu = w.K, w.window.num_imu
    kf = np.array([w.window.imu_kf[q] for q in range(nimu)])
    s = synth.imu_stream(1, K, 34)
    sel = kf  # interval k of the stream spans keyframes k -> k+1
    prm = synth.imu_parameters()
    sb = w.speed_bias().reshape(K, 9)
    args = (s.time_ns, s.readings, s.ranges[sel], s.t0_ns[sel], s.t1_ns[sel])
    built = backend.imu_preintegrate(prm, *args, sb[kf, 3:9])
    for q in range(nimu):
        w.window.imu[q] = built[q]
    sb[kf[1], 3] += 1e-3   # gyro drift above 3e-4
    sb[kf[3], 7] += 0.05   # accelerometer drift above 0.02
    sb[kf[2], 4] += 1e-4   # below both thresholds
    solver = backend.Solver()
    solver.set_windows([w])
    solver.set_imu_samples(prm, *args)
    assert solver.refresh_imu() == 2
    got = solver.read_imu(0, nimu)
    st, ref, cov = oracle.imu_preintegrate(prm, *args, sb[kf, 3:9], covariance=True)
    assert st == 0
    for q in range(nimu):
        if q in (1, 3):
            compare(got[q], ref[q], cov[q])
            assert list(got[q].reference_bias) == list(sb[kf[q], 3:9])
        else:
            assert bytes(got[q]) == bytes(built[q])
    # a second refresh finds nothing left to do
    assert solver.refresh_imu() == 0
    for q in (1, 3):
        w.window.imu[q] = ref[q]
    nr, L = w.retained_dim(), w.L
    ref_step = oracle.step(w.window, nr, L, 1e-4)
    solver.step(1e-4)
    g = solver.read_step(0)
    assert g["status"] == 0 and rel(g["delta"], ref_step["delta"]) < 1e-9


def test_refresh_without_samples_is_rejected(backend):
    from dataclasses import replace
    w = synth.SynthWindow(replace(synth.C1, keyframes=4, landmarks=60), 35)
    solver = backend.Solver()
    solver.set_windows([w])
    with pytest.raises(backend.BackendError) as e:
        solver.refresh_imu()
    assert e.value.code == abi.E_INVALID
