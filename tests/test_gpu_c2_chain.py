"""Configuration 2 as stated, on the device: 10 keyframes, about 3000 landmarks,
IMU factors, 24 + 1 calibration, and a prior chained from five earlier OLD
marginalizations of the preceding sliding windows (each solved and
marginalized on the device, its prior handed to the next window as the
reference's sliding window does, Marginalizer.cpp:284-474,
SlidingWindowManager.cpp:493-700); then the mixed-precision 5-iteration solve.

Bars: every chained prior against the oracle's marginalization of the same
window at the same states (A^T A, A^T r0 within 1e-8, same rank and blocks);
the mixed-precision step dx within 1e-6 of the FP64 step, which is within 1e-9
of the oracle's; the mixed solve's states within 1e-6 of the FP64 solve's with
the same accepted steps; the final window's prior within 1e-8 of the oracle's.
"""
from __future__ import annotations

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _prior_close(got, ref):
    assert got["status"] == 0 and ref["status"] == 0
    assert got["rank"] == ref["rank"] and got["cols"] == ref["cols"]
    assert np.array_equal(got["kinds"], ref["kinds"]) and np.array_equal(got["index"], ref["index"])
    Ag, Ar = got["A"], ref["A"]
    assert rel(Ag.T @ Ag, Ar.T @ Ar) < 1e-8
    assert rel(Ag.T @ got["r0"], Ar.T @ ref["r0"]) < 1e-8


def build_chain(backend, oracle, seed, links=5, iterations=5, check=True):
    """Solves and marginalizes windows 0..links-1 on the device, each prior feeding the next;
    returns the window that carries the chained prior."""
    long = synth.c2_long_window(seed)
    prior = None
    for i in range(links + 1):
        w = synth.SubWindow(long, i, 10)
        if prior is not None:
            w.set_prior(prior, 1)
        if i == links:
            return w
        s = backend.Solver()
        s.set_windows([w])
        s.solve(iterations)
        s.marginalize([0], abi.MARGIN_OLD)
        s.synchronize()
        s.read_states()
        assert s.reports()[0].status in (0, 8)  # CGMLI_E_NO_STEP: a window may keep its state
        prior = s.read_prior(0)
        if check:
            _prior_close(prior, oracle.marginalize_window(w.window, 0, abi.MARGIN_OLD))
        s.close()
        w.store()


@pytest.fixture(scope="module")
def backend():
    from cgmli_slam_b200 import backend as B

    return B


def test_chained_prior_and_mixed_solve(backend, oracle):
    w = build_chain(backend, oracle, seed=21)
    assert w.window.prior_rank > 0 and 2500 <= w.L <= 3500
    nr, L = w.retained_dim(), w.L
    x0 = w.state_vector()
    # one damped step: mixed against FP64 against the oracle
    ref = oracle.step(w.window, nr, L, 1e-4)
    steps = {}
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        s = backend.Solver(precision=prec)
        s.set_windows([w])
        s.step(1e-4)
        steps[prec] = s.read_step(0)
        s.close()
    d64, dmx = steps[abi.PRECISION_FP64]["delta"], steps[abi.PRECISION_MIXED]["delta"]
    assert rel(d64, ref["delta"]) < 1e-9
    assert rel(dmx, d64) < 1e-6
    # 5 iterations in each precision from the same states
    out = {}
    for prec in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        w.set_state_vector(x0)
        s = backend.Solver(precision=prec)
        s.set_windows([w])
        s.solve(5)
        s.synchronize()
        s.read_states()
        out[prec] = (s.reports()[0], w.state_vector())
        s.close()
    r64, x64 = out[abi.PRECISION_FP64]
    rmx, xmx = out[abi.PRECISION_MIXED]
    assert r64.status == rmx.status == 0 and r64.accepted_steps == rmx.accepted_steps
    assert rel(xmx - x0, x64 - x0) < 1e-6
    # the FP64 solve against the oracle's
    w.set_state_vector(x0)
    st, rep = oracle.lm_solve(w.window, 5)
    assert st == 0 and (rep.iterations, rep.accepted_steps) == (r64.iterations, r64.accepted_steps)
    assert rel(w.state_vector() - x0, x64 - x0) < 1e-6
    # the final window's own marginalization after the mixed solve
    w.set_state_vector(xmx)
    s = backend.Solver(precision=abi.PRECISION_MIXED)
    s.set_windows([w])
    s.marginalize([0], abi.MARGIN_OLD)
    got = s.read_prior(0)
    s.close()
    _prior_close(got, oracle.marginalize_window(w.window, 0, abi.MARGIN_OLD))
