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
    return F * (120 + 448) + L * (160 + 8 * (6 * 12 + 7)) + 8 * (3 * Nr * Nr + Npc * Npc + 4 * m * m) + 4096


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
