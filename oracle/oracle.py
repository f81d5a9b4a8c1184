"""ctypes binding of the FP64 CPU oracle (oracle/cgmli_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline arm of bench.py as the checker; never by the product path.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def _pkg():
    name = "cgmli_slam_b200"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, ROOT / "cgmli-slam_b200" / "__init__.py", submodule_search_locations=[str(ROOT / "cgmli-slam_b200")])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


_pkg()
from cgmli_slam_b200 import abi  # noqa: E402
from cgmli_slam_b200.build import build_oracle  # noqa: E402

dp = abi.c_double_p
ip = abi.c_int_p
W = C.POINTER(abi.Window)
_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        L = C.CDLL(str(build_oracle()))
        P = abi._proto
        P(L, "oracle_version", C.c_int, [])
        P(L, "oracle_visual_factor", C.c_int, [W, C.c_int, C.c_int, C.c_int, dp, dp, ip])
        P(L, "oracle_visual_residual_numeric", C.c_int, [W, C.c_int, C.c_int, dp])
        P(L, "oracle_imu_factor", C.c_int, [C.POINTER(abi.FrozenImu), dp, dp, dp, dp, dp, dp])
        P(L, "oracle_pose_plus", None, [dp, dp, dp])
        P(L, "oracle_pose_minus", None, [dp, dp, dp])
        P(L, "oracle_chart_derivative", None, [dp, dp, C.c_int, dp])
        P(L, "oracle_prior_factor", C.c_int, [W, C.c_int, dp, dp])
        P(L, "oracle_linearize", C.c_int, [W, dp, dp, dp, dp, dp])
        P(L, "oracle_step", C.c_int, [W, C.c_double, C.c_int, dp, dp, dp, dp, dp, dp, dp])
        P(L, "oracle_window_cost", C.c_int, [W, dp])
        P(L, "oracle_lm_solve", C.c_int, [W, C.c_int, C.c_double, C.c_int, C.POINTER(abi.SolveReport)])
        P(L, "oracle_lm_solve_batch", C.c_int, [W, C.c_int, C.c_int, C.c_int, C.POINTER(abi.SolveReport)])
        P(L, "oracle_lm_solve_options", C.c_int,
          [W, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, abi.HOST_FACTOR_FN, C.c_void_p, C.c_int, C.POINTER(abi.SolveReport)])
        P(L, "oracle_robust_normal", C.c_int, [C.c_int, C.c_int, dp, dp, C.c_double, dp, dp, dp, dp])
        P(L, "oracle_eigen_sym", C.c_int, [C.c_int, dp, dp, dp])
        P(L, "oracle_psd_solve", C.c_int, [C.c_int, dp, C.c_int, dp, C.c_double, C.c_double, dp])
        P(L, "oracle_marginalize_system", C.c_int,
          [C.c_int, dp, dp, C.c_int, ip, ip, ip, dp, dp, dp, dp, dp])
        P(L, "oracle_marginalize_window", C.c_int,
          [W, C.c_int, C.c_int, ip, ip, ip, ip, ip, dp, dp, dp, dp, dp, dp])
        P(L, "oracle_lm_solve_gated", C.c_int,
          [W, C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(abi.SolveReport), ip, dp, C.POINTER(C.c_ubyte)])
        ll = C.POINTER(C.c_longlong)
        P(L, "oracle_calibration_information", C.c_int, [W, C.c_int, ip, ip, ip, ip, dp, dp])
        P(L, "oracle_marginalize_window_merge", C.c_int,
          [W, C.c_int, C.POINTER(abi.ImuParameters), ll, dp, C.c_int, ip, ll, ll, C.c_double, C.c_int, ip, ip, ip, ip, ip, dp, dp, dp,
           ip, C.POINTER(abi.FrozenImu)])
        P(L, "oracle_imu_preintegrate", C.c_int,
          [C.POINTER(abi.ImuParameters), ll, dp, C.c_int, ip, ll, ll, dp, C.c_int, C.POINTER(abi.FrozenImu), dp])
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(dp)


def visual_factor(win, l, f, derivatives=True):
    r = np.zeros(2)
    J = np.zeros((2, 26))
    flags = np.zeros(2, dtype=np.int32)
    ok = lib().oracle_visual_factor(C.byref(win), l, f, int(derivatives), _p(r), _p(J), flags.ctypes.data_as(ip))
    return bool(ok), r, J, flags


def linearize(win, nr, L):
    H = np.zeros((nr, nr)); g = np.zeros(nr + L); d = np.zeros(L); Cm = np.zeros((L, nr)); cost = np.zeros(1)
    st = lib().oracle_linearize(C.byref(win), _p(H), _p(g), _p(d), _p(Cm), _p(cost))
    return st, H, g, d, Cm, float(cost[0])


def step(win, nr, L, lam, refinement=0):
    delta = np.zeros(nr + L); S = np.zeros((nr, nr)); rhs = np.zeros(nr)
    cost, pred, trial, maxinc = np.zeros(1), np.zeros(1), np.zeros(1), np.zeros(1)
    st = lib().oracle_step(C.byref(win), lam, refinement, _p(delta), _p(S), _p(rhs), _p(cost), _p(pred), _p(trial), _p(maxinc))
    return dict(status=st, delta=delta, S=S, rhs=rhs, cost=float(cost[0]), predicted=float(pred[0]),
                trial_cost=float(trial[0]), max_increment=float(maxinc[0]))


def lm_solve(win, iterations, initial_lambda=1e-4, refinement=0):
    rep = abi.SolveReport()
    st = lib().oracle_lm_solve(C.byref(win), iterations, initial_lambda, refinement, C.byref(rep))
    return st, rep


def host_factor_callback(fn, nr, K, E):
    """Wraps fn(window, trial, poses (K,7), speed_bias (K,9), extrinsics (E,7), td) -> (H, g, cost) or
    cost (trial) in the cgmli_host_factor_fn form (the oracle calls it for one window)."""

    def cb(ctx, w, trial, poses, sb, ext, td, H, g, cost):
        try:
            out = fn(w, bool(trial), np.ctypeslib.as_array(poses, shape=(K, 7)).copy(), np.ctypeslib.as_array(sb, shape=(K, 9)).copy(),
                     np.ctypeslib.as_array(ext, shape=(E, 7)).copy(), float(td[0]))
            if out is None:
                return 1
            if trial:
                cost[0] = float(out)
                return 0
            Hm, gv, c = out
            np.ctypeslib.as_array(H, shape=(nr * nr,))[:] = np.asarray(Hm, dtype=np.float64).reshape(-1)
            np.ctypeslib.as_array(g, shape=(nr,))[:] = np.asarray(gv, dtype=np.float64)
            cost[0] = float(c)
            return 0
        except Exception:  # noqa: BLE001 - a failed evaluation
            return 1

    return abi.HOST_FACTOR_FN(cb)


def lm_solve_options(win, iterations, min_iterations=0, budget_elapsed=False, host=None, nr=0, window_index=0,
                     initial_lambda=1e-4, refinement=0):
    """LM solve in place with the minimum iterations, a budget elapsed from the start (or never) and
    caller-evaluated factors host(window, trial, poses, speed_bias, extrinsics, td) (see backend.Solver.solve_host)."""
    rep = abi.SolveReport()
    cb = host_factor_callback(host, nr, win.num_keyframes, win.num_extrinsics) if host else abi.HOST_FACTOR_FN()
    st = lib().oracle_lm_solve_options(C.byref(win), iterations, initial_lambda, refinement, min_iterations, int(budget_elapsed), cb,
                                       None, window_index, C.byref(rep))
    return st, rep


def window_cost(win):
    c = np.zeros(1)
    st = lib().oracle_window_cost(C.byref(win), _p(c))
    return st, float(c[0])


def robust_normal(J, r, huber):
    J = np.ascontiguousarray(J, dtype=np.float64); r = np.ascontiguousarray(r, dtype=np.float64)
    rows, cols = J.shape
    H = np.zeros((cols, cols)); g = np.zeros(cols); cost = np.zeros(1); rss = np.zeros(1)
    lib().oracle_robust_normal(rows, cols, _p(J), _p(r), huber, _p(H), _p(g), _p(cost), _p(rss))
    return H, g, float(cost[0]), float(rss[0])


def eigen_sym(H):
    n = H.shape[0]
    Hc = np.ascontiguousarray(H, dtype=np.float64)
    ev = np.zeros(n); V = np.zeros((n, n))
    st = lib().oracle_eigen_sym(n, _p(Hc), _p(ev), _p(V))
    return st, ev, V


def psd_solve(H, rhs, abs_cut=1e-12, rel_cut=1e-9):
    H = np.ascontiguousarray(H, dtype=np.float64)
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    if rhs.ndim == 1:
        rhs = rhs[:, None]
    x = np.zeros_like(rhs)
    st = lib().oracle_psd_solve(H.shape[0], _p(H), rhs.shape[1], _p(rhs), abs_cut, rel_cut, _p(x))
    return st, x


def marginalize_system(H, b, blocks):
    """blocks: list of (size, eliminate, landmark)."""
    n = H.shape[0]
    H = np.ascontiguousarray(H, dtype=np.float64); b = np.ascontiguousarray(b, dtype=np.float64)
    desc = np.array([v for bl in blocks for v in bl], dtype=np.int32)
    rank, nr = np.zeros(1, np.int32), np.zeros(1, np.int32)
    Hp = np.zeros(n * n); bp = np.zeros(n); A = np.zeros(n * n); r0 = np.zeros(n); stats = np.zeros(3)
    st = lib().oracle_marginalize_system(n, _p(H), _p(b), len(blocks), desc.ctypes.data_as(ip), rank.ctypes.data_as(ip),
                                         nr.ctypes.data_as(ip), _p(Hp), _p(bp), _p(A), _p(r0), _p(stats))
    k, m = int(rank[0]), int(nr[0])
    return dict(status=st, rank=k, nr=m, H=Hp[:m * m].reshape(m, m), b=bp[:m], A=A[:k * m].reshape(k, m), r0=r0[:k],
                eliminated_reduction=stats[0], cutoff=stats[1], new_reference_norm=stats[2])


def marginalize_window(win, victim, policy=abi.MARGIN_OLD):
    rank, cols, nb = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32)
    st = lib().oracle_marginalize_window(C.byref(win), victim, policy, rank.ctypes.data_as(ip), cols.ctypes.data_as(ip),
                                         nb.ctypes.data_as(ip), None, None, None, None, None, None, None, None)
    if st != 0:
        return dict(status=st)
    k, m, b = int(rank[0]), int(cols[0]), int(nb[0])
    kinds, idx = np.zeros(b, np.int32), np.zeros(b, np.int32)
    ref = np.zeros(7 * b + 9 * b); Hp = np.zeros(m * m); bp = np.zeros(m); A = np.zeros(k * m); r0 = np.zeros(k)
    form = np.zeros(4)
    st = lib().oracle_marginalize_window(C.byref(win), victim, policy, rank.ctypes.data_as(ip), cols.ctypes.data_as(ip),
                                         nb.ctypes.data_as(ip), kinds.ctypes.data_as(ip), idx.ctypes.data_as(ip), _p(ref),
                                         _p(Hp), _p(bp), _p(A), _p(r0), _p(form))
    return dict(status=st, rank=k, cols=m, kinds=kinds, index=idx, reference=ref, H=Hp.reshape(m, m), b=bp,
                A=A.reshape(k, m), r0=r0, robust_cost=form[0], rss=form[1], eliminated_reduction=form[2], cutoff=form[3])


def lm_solve_batch(windows_array, count, iterations, threads):
    reps = (abi.SolveReport * count)()
    st = lib().oracle_lm_solve_batch(windows_array, count, iterations, threads, reps)
    return st, reps


def imu_preintegrate(params, time_ns, readings, ranges, t0_ns, t1_ns, bias, covariance=False):
    """Frozen IMU factors of count intervals (see cgmli_imu_preintegrate);
    with covariance=True also the (count, 15, 15) preintegrated covariances."""
    ll = C.POINTER(C.c_longlong)
    time_ns = np.ascontiguousarray(time_ns, dtype=np.int64)
    readings = np.ascontiguousarray(readings, dtype=np.float64)
    ranges = np.ascontiguousarray(ranges, dtype=np.int32)
    t0_ns = np.ascontiguousarray(t0_ns, dtype=np.int64)
    t1_ns = np.ascontiguousarray(t1_ns, dtype=np.int64)
    bias = np.ascontiguousarray(bias, dtype=np.float64)
    count = len(t0_ns)
    out = (abi.FrozenImu * max(count, 1))()
    cov = np.zeros((max(count, 1), 15, 15)) if covariance else None
    st = lib().oracle_imu_preintegrate(C.byref(params), time_ns.ctypes.data_as(ll), _p(readings), len(time_ns),
                                       ranges.ctypes.data_as(ip), t0_ns.ctypes.data_as(ll), t1_ns.ctypes.data_as(ll),
                                       _p(bias), count, out, _p(cov))
    return (st, out, cov[:count]) if covariance else (st, out)


def lm_solve_gated(win, iterations, threshold=9.210340371976184, max_refits=3, pre_gate=True):
    """Gated LM solve in place; (status, report, gate dict, rejected mask)."""
    rep = abi.SolveReport()
    gate = np.zeros(5, dtype=np.int32)
    nis = np.zeros(2)
    mask = np.zeros(max(win.num_observations, 1), dtype=np.uint8)
    st = lib().oracle_lm_solve_gated(C.byref(win), iterations, threshold, max_refits, int(pre_gate), C.byref(rep),
                                     gate.ctypes.data_as(ip), _p(nis), mask.ctypes.data_as(C.POINTER(C.c_ubyte)))
    g = dict(passes=int(gate[0]), rejected_pre=int(gate[1]), evaluated=int(gate[2]), rejected_last=int(gate[3]),
             rejected_total=int(gate[4]), nis_sum=float(nis[0]), nis_max=float(nis[1]))
    return st, rep, g, mask[:win.num_observations]


def marginalize_window_merge(win, victim, params, time_ns, readings, ranges, t0_ns, t1_ns, max_interval=10.0, max_samples=10000):
    """SECOND_NEW marginalization with the IMU merge; the prior (as
    marginalize_window, without H/b) plus 'merge' (CGMLI_IMU_MERGE_*) and
    'merged' (the re-integrated factor or None)."""
    ll = C.POINTER(C.c_longlong)
    time_ns = np.ascontiguousarray(time_ns, dtype=np.int64)
    readings = np.ascontiguousarray(readings, dtype=np.float64)
    ranges = np.ascontiguousarray(ranges, dtype=np.int32)
    t0_ns = np.ascontiguousarray(t0_ns, dtype=np.int64)
    t1_ns = np.ascontiguousarray(t1_ns, dtype=np.int64)
    rank, cols, nb, state = (np.zeros(1, np.int32) for _ in range(4))
    merged = abi.FrozenImu()
    args = (C.byref(win), victim, C.byref(params), time_ns.ctypes.data_as(ll), _p(readings), len(time_ns),
            ranges.ctypes.data_as(ip), t0_ns.ctypes.data_as(ll), t1_ns.ctypes.data_as(ll), max_interval, max_samples,
            rank.ctypes.data_as(ip), cols.ctypes.data_as(ip), nb.ctypes.data_as(ip))
    st = lib().oracle_marginalize_window_merge(*args, None, None, None, None, None, state.ctypes.data_as(ip), C.byref(merged))
    if st != 0:
        return dict(status=st)
    k, m, b = int(rank[0]), int(cols[0]), int(nb[0])
    kinds, idx = np.zeros(b, np.int32), np.zeros(b, np.int32)
    ref = np.zeros(9 * b + 1); A = np.zeros(k * m); r0 = np.zeros(k)
    st = lib().oracle_marginalize_window_merge(*args, kinds.ctypes.data_as(ip), idx.ctypes.data_as(ip), _p(ref), _p(A), _p(r0),
                                               state.ctypes.data_as(ip), C.byref(merged))
    return dict(status=st, rank=k, cols=m, kinds=kinds, index=idx, reference=ref, A=A.reshape(k, m), r0=r0,
                merge=int(state[0]), merged=merged if int(state[0]) == abi.IMU_MERGE_REINTEGRATED else None)


def calibration_information(win, include_prior=False):
    """Conditional calibration information of a window: blocks, matrix, eigenvalues."""
    size, nb = np.zeros(1, np.int32), np.zeros(1, np.int32)
    st = lib().oracle_calibration_information(C.byref(win), int(include_prior), size.ctypes.data_as(ip), nb.ctypes.data_as(ip),
                                              None, None, None, None)
    if st != 0:
        return dict(status=st)
    n, b = int(size[0]), int(nb[0])
    kinds, idx = np.zeros(max(b, 1), np.int32), np.zeros(max(b, 1), np.int32)
    cond, ev = np.zeros(max(n * n, 1)), np.zeros(max(n, 1))
    st = lib().oracle_calibration_information(C.byref(win), int(include_prior), size.ctypes.data_as(ip), nb.ctypes.data_as(ip),
                                              kinds.ctypes.data_as(ip), idx.ctypes.data_as(ip), _p(cond), _p(ev))
    return dict(status=st, kinds=kinds[:b], index=idx[:b], conditional=cond[:n * n].reshape(n, n), eigenvalues=ev[:n])
