"""CPU tests of the IMU preintegration oracle (ImuError::redoPreintegration,
src/factor/ImuError.cpp:254-462) against the reference's known answers and
derivative checks, and of the host-side checks of cgmli_imu_preintegrate."""
from __future__ import annotations

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth


def mat(f, name):
    return np.array(getattr(f, name)).reshape(3, 3, order="F")


def whitening(f):
    return np.array(f.whitening).reshape(15, 15, order="F")


def qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by + ay * bw + az * bx - ax * bz,
                     aw * bz + az * bw + ax * by - ay * bx, aw * bw - ax * bx - ay * by - az * bz])


def qlog(q):
    n = np.linalg.norm(q[:3])
    return 2 * np.arctan2(n, q[3]) * q[:3] / n if n > 0 else 2 * q[:3]


def stationary_stream(end_s=1.0):
    """samples() of src/pipeline/tests/NativeSlamRegression.cpp:126-130: 200 Hz,
    zero rotation rate, specific force (0, 0, 9.81)."""
    n = int(end_s * 200) + 1
    t = (np.arange(n, dtype=np.int64) * 1_000_000_000) // 200
    readings = np.tile([0.0, 0.0, 0.0, 0.0, 0.0, 9.81], (n, 1))
    return t, readings


# parameters() of NativeSlamRegression.cpp:112-125 (IMU part)
TEST_IMU = dict(sigma_g_c=0.002, sigma_a_c=0.02, sigma_gw_c=0.0002, sigma_aw_c=0.002, g_max=100, a_max=100, g=9.81,
                max_sample_gap=0.05)


def test_stationary_known_answer(oracle):
    """bodyImuJacobianAndFrozenCost (NativeSlamRegression.cpp:601-612) integrates
    a stationary sensor over [0.5, 0.55] s; for constant readings the trapezoid
    recursion is exact: no rotation, C_integral = T I, double integral T^2/2 I,
    velocity T g, position T^2/2 g, d alpha / d b_g = T I, d v / d b_g = T^2/2 [g]x."""
    t, rd = stationary_stream()
    prm = synth.imu_parameters(**TEST_IMU)
    st, f = oracle.imu_preintegrate(prm, t, rd, [[0, len(t)]], [500_000_000], [550_000_000], np.zeros((1, 6)))
    assert st == 0
    f = f[0]
    T = 0.05
    g = np.array([0.0, 0.0, 9.81])
    assert np.allclose(f.delta_quaternion, [0, 0, 0, 1], atol=0)
    assert np.allclose(mat(f, "velocity_accel"), T * np.eye(3), rtol=0, atol=1e-15)
    assert np.allclose(mat(f, "position_accel"), 0.5 * T * T * np.eye(3), rtol=0, atol=1e-16)
    assert np.allclose(f.delta_velocity, T * g, rtol=1e-14, atol=1e-15)
    assert np.allclose(f.delta_position, 0.5 * T * T * g, rtol=1e-14, atol=1e-16)
    assert np.allclose(mat(f, "rotation_gyro"), T * np.eye(3), rtol=0, atol=1e-15)
    gx = np.array([[0, -g[2], g[1]], [g[2], 0, -g[0]], [-g[1], g[0], 0]])
    assert np.allclose(mat(f, "velocity_gyro"), 0.5 * T * T * gx, rtol=1e-13, atol=1e-16)
    assert f.duration == pytest.approx(T, rel=1e-15)
    assert f.gravity == 9.81
    assert list(f.gyros) == [0.0] * 6
    assert list(f.reference_bias) == [0.0] * 6


@pytest.mark.parametrize("on_sample", [False, True])
def test_whitening_inverts_covariance(oracle, on_sample):
    """W = diag(1/sqrt(lambda)) U^T (PseudoInverse::symmSqrtU): W P W^T = I."""
    s = synth.imu_stream(3, 6, 5, on_sample=on_sample)
    st, fz, cov = oracle.imu_preintegrate(synth.imu_parameters(), s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias,
                                          covariance=True)
    assert st == 0
    for i in range(s.count):
        W = whitening(fz[i])
        assert np.abs(W @ cov[i] @ W.T - np.eye(15)).max() < 1e-12
        assert np.allclose(cov[i], cov[i].T, rtol=0, atol=0)
        # rows of W ordered by ascending eigenvalue: row norms descend
        norms = np.linalg.norm(W, axis=1)
        assert np.all(np.diff(norms) <= 1e-12 * norms[0])


def test_bias_jacobians_match_central_differences(oracle):
    """The five bias Jacobians are the derivatives of the discrete recursion:
    Delta_q(b) ~ Exp(-J_alpha db_g) Delta_q, Delta_v(b) ~ Delta_v + J_v db_g - C_int db_a,
    Delta_p(b) ~ Delta_p + J_p db_g - C_dint db_a (ImuError.cpp:899-933)."""
    s = synth.imu_stream(2, 4, 11)
    prm = synth.imu_parameters()
    i = 2
    st, fz = oracle.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    assert st == 0
    base = fz[i]
    h = 1e-6
    for c in range(6):
        outs = []
        for sgn in (1, -1):
            b = s.bias[i:i + 1].copy()
            b[0, c] += sgn * h
            st, f2 = oracle.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges[i:i + 1], s.t0_ns[i:i + 1], s.t1_ns[i:i + 1], b)
            assert st == 0
            outs.append(f2[0])
        dv = (np.array(outs[0].delta_velocity) - np.array(outs[1].delta_velocity)) / (2 * h)
        dp = (np.array(outs[0].delta_position) - np.array(outs[1].delta_position)) / (2 * h)
        qm = np.array(outs[1].delta_quaternion) * [-1, -1, -1, 1]
        da = qlog(qmul(np.array(outs[0].delta_quaternion), qm)) / (2 * h)
        if c < 3:
            for got, ref in ((dv, mat(base, "velocity_gyro")[:, c]), (dp, mat(base, "position_gyro")[:, c]),
                             (-da, mat(base, "rotation_gyro")[:, c])):
                assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
        else:
            k = c - 3
            for got, ref in ((-dv, mat(base, "velocity_accel")[:, k]), (-dp, mat(base, "position_accel")[:, k])):
                assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()
            assert np.abs(da).max() == 0.0


def test_gyro_readings_at_interval_ends(oracle):
    """gyroAt (BodyImuFactor.cpp:29-38): linear interpolation between the samples
    around each end."""
    s = synth.imu_stream(1, 3, 4)
    st, fz = oracle.imu_preintegrate(synth.imu_parameters(), s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    assert st == 0
    for i in range(s.count):
        for end, t in enumerate((s.t0_ns[i], s.t1_ns[i])):
            k = int(np.searchsorted(s.time_ns, t))
            a = (t - s.time_ns[k - 1]) / (s.time_ns[k] - s.time_ns[k - 1])
            ref = (1 - a) * s.readings[k - 1, :3] + a * s.readings[k, :3]
            assert np.allclose(fz[i].gyros[3 * end:3 * end + 3], ref, rtol=1e-14, atol=1e-17)


def test_saturation_inflates_noise(oracle):
    """A reading above g_max / a_max scales that noise by 100 (ImuError.cpp:333-354)."""
    s = synth.imu_stream(1, 3, 6)
    prm = synth.imu_parameters()
    st, _, cov = oracle.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias, covariance=True)
    rd = s.readings.copy()
    b, e = s.ranges[0]
    rd[(b + e) // 2, 0] = 10.0   # gyro above 7.8 rad/s
    rd[(b + e) // 2, 5] = 200.0  # accelerometer above 176 m/s^2
    st2, _, cov2 = oracle.imu_preintegrate(prm, s.time_ns, rd, s.ranges, s.t0_ns, s.t1_ns, s.bias, covariance=True)
    assert st == 0 and st2 == 0
    # the sample enters two of the ~60 steps, each with 100x the white noise
    assert np.trace(cov2[0][3:6, 3:6]) > 3 * np.trace(cov[0][3:6, 3:6])
    assert np.trace(cov2[0][6:9, 6:9]) > 3 * np.trace(cov[0][6:9, 6:9])
    assert np.allclose(cov2[1], cov[1])  # the other interval has no saturated sample


def test_invalid_intervals(oracle):
    """validImuInterval (BodyImuFactor.cpp:10-28): bracketing, increasing times,
    finite readings and the sample-gap limit."""
    s = synth.imu_stream(1, 3, 2)
    prm = synth.imu_parameters()
    args = lambda **kw: {**dict(time_ns=s.time_ns, readings=s.readings, ranges=s.ranges, t0_ns=s.t0_ns, t1_ns=s.t1_ns,
                                bias=s.bias), **kw}
    assert oracle.imu_preintegrate(prm, **args())[0] == 0
    late = s.t0_ns.copy(); late[1] = s.time_ns[s.ranges[1][0]] - 1  # starts before the range
    assert oracle.imu_preintegrate(prm, **args(t0_ns=late))[0] == abi.E_INVALID
    t = s.time_ns.copy(); b = s.ranges[0][0]; t[b + 5] = t[b + 4]      # repeated time stamp
    assert oracle.imu_preintegrate(prm, **args(time_ns=t))[0] == abi.E_INVALID
    rd = s.readings.copy(); rd[b + 7, 2] = np.nan
    assert oracle.imu_preintegrate(prm, **args(readings=rd))[0] == abi.E_INVALID
    tight = synth.imu_parameters(max_sample_gap=0.004)                 # 5 ms sampling
    assert oracle.imu_preintegrate(tight, **args())[0] == abi.E_INVALID
    backwards = s.t1_ns.copy(); backwards[0] = s.t0_ns[0]
    assert oracle.imu_preintegrate(prm, **args(t1_ns=backwards))[0] == abi.E_INVALID
