"""Served mode on the GPU: requests batched continuously give the same result
as each window solved alone (states within 1e-8 relative - only the order of
FP64 reductions differs - and the marginal prior's A^T A / A^T r0 within
1e-8), whatever batches the scheduler forms."""
from __future__ import annotations

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


def _alone(backend, w, victim, iterations, precision=abi.PRECISION_FP64):
    s = backend.Solver(precision=precision)
    s.set_windows([w])
    s.solve(iterations)
    prior = None
    if victim >= 0:
        s.marginalize([victim], abi.MARGIN_OLD)
        prior = s.read_prior(0)
    s.synchronize()
    s.read_states()
    rep = s.reports()[0]
    s.close()
    return w.state_vector(), rep, prior


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("budget", [40 << 30, 1])  # 1 byte: every batch holds a single window
def test_served_equals_alone(backend, budget, precision):
    """Also in mixed precision: a window's mixed linearization does not depend on
    its batch neighbours, so the same bars hold."""
    n, iterations = 10, 1
    alone_windows = synth.make_windows("c4", n, seed=321)
    served_windows = synth.make_windows("c4", n, seed=321)
    x0 = [w.state_vector() for w in served_windows]
    victims = [0 if i % 3 else -1 for i in range(n)]
    ref = [_alone(backend, w, v, iterations, precision) for w, v in zip(alone_windows, victims)]
    server = backend.Server(iterations=iterations, policy=abi.MARGIN_OLD, max_batch_windows=4, memory_budget_bytes=budget,
                            precision=precision)
    tickets = [server.submit(w, v) for w, v in zip(served_windows, victims)]
    for i, t in enumerate(tickets):
        rep, latency = server.poll(t, wait=True)
        assert rep.status == 0 and latency > 0
        x_ref, rep_ref, prior_ref = ref[i]
        assert rep.iterations == rep_ref.iterations and rep.accepted_steps == rep_ref.accepted_steps
        assert rel(served_windows[i].state_vector() - x0[i], x_ref - x0[i]) < 1e-8
        if victims[i] >= 0:
            got = server.read_prior(t)
            assert got["status"] == 0 and got["rank"] == prior_ref["rank"] and got["cols"] == prior_ref["cols"]
            Ag, Ar = got["A"], prior_ref["A"]
            assert rel(Ag.T @ Ag, Ar.T @ Ar) < 1e-8
            assert rel(Ag.T @ got["r0"], Ar.T @ prior_ref["r0"]) < 1e-8
        server.release(t)
    server.close()


def test_served_deterministic_equals_alone_bitwise(backend):
    """With deterministic sums on both sides, every request's solved states and report
    are bit for bit those of its window solved alone, whatever batches the scheduler
    forms (batches of up to 4 windows here, mixed precision, 3 iterations)."""
    n, iterations = 10, 3
    alone_windows = synth.make_windows("c4", n, seed=654)
    served_windows = synth.make_windows("c4", n, seed=654)
    victims = [0 if i % 3 else -1 for i in range(n)]
    ref = []
    for w in alone_windows:
        s = backend.Solver(precision=abi.PRECISION_MIXED)
        s.set_tuning(deterministic=1)
        s.set_windows([w])
        s.solve(iterations)
        s.synchronize()
        s.read_states()
        r = s.reports()[0]
        ref.append((w.state_vector().copy(), (r.iterations, r.accepted_steps, r.status, r.final_cost)))
        s.close()
    server = backend.Server(iterations=iterations, policy=abi.MARGIN_OLD, max_batch_windows=4, precision=abi.PRECISION_MIXED,
                            deterministic=True)
    tickets = [server.submit(w, v) for w, v in zip(served_windows, victims)]
    for i, t in enumerate(tickets):
        rep, _ = server.poll(t, wait=True)
        assert (rep.iterations, rep.accepted_steps, rep.status, rep.final_cost) == ref[i][1]
        assert np.array_equal(served_windows[i].state_vector(), ref[i][0])
        server.release(t)
    server.close()


def test_invalid_request_rejected_at_submit(backend):
    w = synth.SynthWindow(synth.C1, 4)
    arr = synth.window_array([w])
    arr[0].num_keyframes = 2  # observations now reference missing keyframes
    server = backend.Server()
    with pytest.raises(backend.BackendError) as e:
        server.submit(arr[0])
    assert e.value.code == 1
    server.close()


def test_served_gated_equals_alone(backend):
    """With nis_threshold set, every request is solved with the NIS gate and
    outlier refits; its rejected factors and states equal the window's gated
    solve alone."""
    n, iterations = 5, 8
    alone_windows = synth.make_windows("c4", n, seed=95)
    served_windows = synth.make_windows("c4", n, seed=95)
    alone = []
    for w in alone_windows:
        s = backend.Solver()
        s.set_windows([w])
        s.solve_gated(iterations, pre_gate=False)
        s.synchronize()
        s.read_states()
        alone.append((w.state_vector(), s.read_gate(0)[1]))
        s.close()
    x0 = [w.state_vector() for w in served_windows]
    srv = backend.Server(iterations=iterations, nis_threshold=9.210340371976184, max_refits=3, pre_gate=False)
    tickets = [srv.submit(w) for w in served_windows]
    for t, w, x, (xa, ma) in zip(tickets, served_windows, x0, alone):
        rep, _ = srv.poll(t)
        assert rep.status == 0
        g, m = srv.read_gate(t, w.window.num_observations)
        assert np.array_equal(m, ma) and g.rejected_total == int(ma.sum())
        # 8 iterations and refits: the run-to-run order of the FP64 atomic sums, which
        # differs between any two solves of the same window, grows to about 1e-8 here
        assert rel(w.state_vector() - x, xa - x) < 1e-7
        srv.release(t)
    srv.close()


def _footprint(win):
    """The server's per-window device estimate (server.cpp footprint())."""
    F, L, K = win.num_observations, win.num_landmarks, win.num_keyframes
    ncal = (6 * win.num_extrinsics if win.estimate_extrinsics else 0) + (1 if win.estimate_td else 0)
    Nr, Npc, m = 15 * K + ncal, 6 * K + ncal, 15 * K + 6 * win.num_extrinsics + 1
    return F * (120 + 108 + 448) + L * (160 + 8 * (6 * 12 + 7)) + 8 * (3 * Nr * Nr + Npc * Npc + 4 * m * m) + 4096


def test_two_solvers_stay_within_the_memory_budget(backend):
    """Both solvers keep their device arrays between batches; admission limits each batch to half
    of memory_budget_bytes (growth headroom included), so what the two hold together stays within
    the budget while batches of several windows still form."""
    windows = synth.make_windows("c4", 16, seed=404)
    biggest = max(_footprint(w.window) for w in windows)
    budget = int(2 * 1.5 * 3 * biggest)
    server = backend.Server(iterations=1, max_batch_windows=16, memory_budget_bytes=budget)
    tickets = [server.submit(w, 0) for w in windows]
    for t in tickets:
        rep, _ = server.poll(t)
        assert rep.status == 0
        server.release(t)
    held = server.device_bytes()
    server.close()
    assert 0 < held <= budget


def _imu_window(backend, seed):
    """A window whose IMU factors are preintegrated on the device from a sample
    stream, with three keyframes' biases then moved (two past the refresh
    thresholds); returns the window and the samples of its factors."""
    from dataclasses import replace
    w = synth.SynthWindow(replace(synth.C1, keyframes=6, landmarks=200), seed)
    K, nimu = w.K, w.window.num_imu
    kf = np.array([w.window.imu_kf[q] for q in range(nimu)])
    s = synth.imu_stream(1, K, seed + 1)
    prm = synth.imu_parameters()
    sb = w.speed_bias().reshape(K, 9)
    args = (s.time_ns, s.readings, s.ranges[kf], s.t0_ns[kf], s.t1_ns[kf])
    built = backend.imu_preintegrate(prm, *args, sb[kf, 3:9])
    for q in range(nimu):
        w.window.imu[q] = built[q]
    sb[kf[1], 3] += 1e-3
    sb[kf[3], 7] += 0.05
    sb[kf[2], 4] += 1e-4
    return w, prm, args


def test_served_imu_refresh_equals_the_solver(backend):
    """A request with IMU samples: the server refreshes the drifted factors before
    the solve exactly as cgmli_solver_set_imu_samples + _refresh_imu do, and a
    request without samples in the same server keeps its factors as given."""
    w1, prm, args = _imu_window(backend, 61)
    w2, _, _ = _imu_window(backend, 61)
    plain, _, _ = _imu_window(backend, 63)
    nimu = w1.window.num_imu
    s = backend.Solver()
    s.set_windows([w1])
    s.set_imu_samples(prm, *args)
    assert s.refresh_imu() == 2
    ref_imu = s.read_imu(0, nimu)
    s.solve(3)
    s.synchronize()
    s.read_states()
    x_ref = w1.state_vector()
    s.close()
    x_plain0 = plain.state_vector()
    x_plain, _, _ = _alone(backend, _imu_window(backend, 63)[0], -1, 3)
    srv = backend.Server(iterations=3, imu_params=prm)
    t1 = srv.submit_request(w2, -1, imu=args)
    t2 = srv.submit_request(plain, -1)
    rep1, _ = srv.poll(t1)
    rep2, _ = srv.poll(t2)
    assert rep1.status == 0 and rep2.status == 0
    got, refreshed = srv.read_imu(t1, nimu)
    assert refreshed == 2
    assert all(bytes(a) == bytes(b) for a, b in zip(got, ref_imu))
    # another window may share the batch: the FP64 sums of a window add in launch
    # order, and three iterations of a weakly constrained window carry that
    # difference to about 1e-8 (the step bar of the configuration is 1e-6)
    assert rel(w2.state_vector(), x_ref) < 1e-7
    assert rel(plain.state_vector() - x_plain0, x_plain - x_plain0) < 1e-7
    with pytest.raises(backend.BackendError):
        srv.read_imu(t2, nimu)  # that request brought no samples
    srv.close()


def test_served_calibration_information_equals_the_solver(backend):
    """A request for the calibration information (with the prior) and a
    marginalization: the server reads the information back before the
    marginalization reuses the device buffers; both equal the solver's."""
    from dataclasses import replace
    spec = replace(synth.C2, landmarks=400)
    w1, w2 = synth.SynthWindow(spec, 71), synth.SynthWindow(spec, 71)
    s = backend.Solver()
    s.set_windows([w1])
    s.solve(2)
    s.calibration_information(True)
    ref = s.read_calibration_information(0)
    s.marginalize([0], abi.MARGIN_OLD)
    ref_prior = s.read_prior(0)
    s.close()
    assert ref["status"] == 0
    srv = backend.Server(iterations=2, calibration_include_prior=True)
    t = srv.submit_request(w2, 0, calibration=True)
    rep, _ = srv.poll(t)
    assert rep.status == 0
    got = srv.read_calibration_information(t)
    assert got["status"] == 0 and np.array_equal(got["kinds"], ref["kinds"])
    # both at states solved on their own: those agree to the FP64 reduction order (1e-8)
    assert rel(got["conditional"], ref["conditional"]) < 1e-8
    prior = srv.read_prior(t)
    A, Ar = prior["A"], ref_prior["A"]
    assert prior["rank"] == ref_prior["rank"] and rel(A.T @ A, Ar.T @ Ar) < 1e-8
    srv.close()


def test_served_imu_merge_equals_the_solver(backend):
    """A server with the IMU-merge policy: a request with IMU samples and the
    second-newest keyframe as victim gets the same merged factor and the same prior
    as the solver given the same samples (refresh, solve, merge); a request without
    samples in the same server keeps the Schur bridge."""
    w1, prm, args = _imu_window(backend, 65)
    w2, _, _ = _imu_window(backend, 65)
    plain, _, _ = _imu_window(backend, 67)
    v = w1.K - 2
    s = backend.Solver()
    s.set_windows([w1])
    s.set_imu_samples(prm, *args)
    s.refresh_imu()
    s.solve(2)
    s.marginalize([v], abi.MARGIN_SECOND_NEW_IMU_MERGE)
    ref_prior = s.read_prior(0)
    ref_state, ref_f = s.read_merged_imu(0)
    s.close()
    assert ref_state == abi.IMU_MERGE_REINTEGRATED
    srv = backend.Server(iterations=2, imu_params=prm, policy=abi.MARGIN_SECOND_NEW_IMU_MERGE)
    t1 = srv.submit_request(w2, v, imu=args)
    t2 = srv.submit_request(plain, plain.K - 2)
    rep1, _ = srv.poll(t1)
    rep2, _ = srv.poll(t2)
    assert rep1.status == 0 and rep2.status == 0
    state, f = srv.read_merged_imu(t1)
    assert state == abi.IMU_MERGE_REINTEGRATED
    for name in ("delta_quaternion", "delta_velocity", "delta_position", "rotation_gyro", "velocity_gyro", "position_gyro",
                 "velocity_accel", "position_accel", "gyros", "reference_bias"):
        assert rel(getattr(f, name), getattr(ref_f, name)) < 1e-7, name  # the solved bias it is taken at: 1e-8 drift
    got = srv.read_prior(t1)
    A, Ar = got["A"], ref_prior["A"]
    assert got["rank"] == ref_prior["rank"] and got["cols"] == ref_prior["cols"]
    assert rel(A.T @ A, Ar.T @ Ar) < 1e-7
    assert srv.read_merged_imu(t2)[0] == abi.IMU_MERGE_BRIDGE
    srv.close()
