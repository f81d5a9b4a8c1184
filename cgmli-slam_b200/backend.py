"""Python binding of the B200 backend solver C ABI (include/cgmli_backend.h).

The compute runs in ``lib/libcgmli_backend.so``; there is no Python or CPU
fallback: if the library cannot be loaded the import fails loudly.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .build import build_backend

_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = build_backend()
        _LIB = abi.declare_backend(C.CDLL(str(path)))
    return _LIB


class BackendError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {abi.ERRORS.get(code, code)} ({lib().cgmli_last_error().decode()})")


def _check(code: int, where: str) -> None:
    if code != abi.OK:
        raise BackendError(code, where)


def _p(a):
    return a.ctypes.data_as(abi.c_double_p)


class Solver:
    """Batched window solver on one GPU (one CUDA stream)."""

    def __init__(self, device: int = 0, precision: int = abi.PRECISION_FP64, refinement: int = 0,
                 initial_lambda: float = 1e-4, min_iterations: int = 0, time_budget_s: float = 0.0):
        opt = abi.SolverOptions()
        lib().cgmli_default_options(C.byref(opt))
        opt.precision = precision
        opt.refinement_steps = refinement
        opt.initial_lambda = initial_lambda
        opt.min_iterations = min_iterations
        opt.time_budget_s = time_budget_s
        h = C.c_void_p()
        _check(lib().cgmli_solver_create(device, C.byref(opt), C.byref(h)), "cgmli_solver_create")
        self._h = h
        self._windows = None
        self.count = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().cgmli_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_windows(self, windows) -> None:
        arr = windows if isinstance(windows, C.Array) else _window_array(windows)
        self._windows = arr
        self.count = len(arr)
        _check(lib().cgmli_solver_set_windows(self._h, arr, len(arr)), "cgmli_solver_set_windows")

    def upload_states(self) -> None:
        _check(lib().cgmli_solver_upload_states(self._h, self._windows, self.count), "cgmli_solver_upload_states")

    def solve(self, iterations: int) -> None:
        _check(lib().cgmli_solver_solve(self._h, iterations), "cgmli_solver_solve")

    def synchronize(self) -> None:
        _check(lib().cgmli_solver_synchronize(self._h), "cgmli_solver_synchronize")

    def read_states(self) -> None:
        _check(lib().cgmli_solver_read_states(self._h, self._windows, self.count), "cgmli_solver_read_states")

    def reports(self) -> list[abi.SolveReport]:
        reps = (abi.SolveReport * self.count)()
        _check(lib().cgmli_solver_read_reports(self._h, reps, self.count), "cgmli_solver_read_reports")
        return list(reps)

    def solve_gated(self, iterations: int, nis_threshold: float = 9.210340371976184, max_refits: int = 3, pre_gate: bool = True):
        _check(lib().cgmli_solver_solve_gated(self._h, iterations, nis_threshold, max_refits, int(pre_gate)),
               "cgmli_solver_solve_gated")

    def read_gate(self, w: int):
        """(GateReport, rejected mask over the window's observations)."""
        rep = abi.GateReport()
        n = self._windows[w].num_observations
        mask = np.zeros(max(n, 1), dtype=np.uint8)
        _check(lib().cgmli_solver_read_gate(self._h, w, C.byref(rep), mask.ctypes.data_as(C.POINTER(C.c_ubyte))),
               "cgmli_solver_read_gate")
        return rep, mask[:n]

    def calibration_information(self, include_prior: bool = False) -> None:
        _check(lib().cgmli_solver_calibration_information(self._h, int(include_prior)), "cgmli_solver_calibration_information")

    def read_calibration_information(self, w: int) -> dict:
        """Conditional calibration information of window w: blocks, matrix, eigenvalues."""
        size, nb = C.c_int(), C.c_int()
        code = lib().cgmli_solver_read_calibration_information(self._h, w, C.byref(size), C.byref(nb), None, None, None, None)
        if code != 0:
            return dict(status=code)
        n, b = size.value, nb.value
        kinds, idx = np.zeros(max(b, 1), np.int32), np.zeros(max(b, 1), np.int32)
        cond, ev = np.zeros(max(n * n, 1)), np.zeros(max(n, 1))
        code = lib().cgmli_solver_read_calibration_information(self._h, w, C.byref(size), C.byref(nb), kinds.ctypes.data_as(abi.c_int_p),
                                                               idx.ctypes.data_as(abi.c_int_p), _p(cond), _p(ev))
        return dict(status=code, kinds=kinds[:b], index=idx[:b], conditional=cond[:n * n].reshape(n, n), eigenvalues=ev[:n])

    def set_imu_merge_limits(self, max_interval_s: float = 10.0, max_samples: int = 10000) -> None:
        _check(lib().cgmli_solver_set_imu_merge_limits(self._h, max_interval_s, max_samples), "cgmli_solver_set_imu_merge_limits")

    def read_merged_imu(self, w: int):
        """(outcome CGMLI_IMU_MERGE_*, merged factor or None) of window w."""
        state = C.c_int()
        f = abi.FrozenImu()
        _check(lib().cgmli_solver_read_merged_imu(self._h, w, C.byref(state), C.byref(f)), "cgmli_solver_read_merged_imu")
        return state.value, (f if state.value == abi.IMU_MERGE_REINTEGRATED else None)

    def set_imu_samples(self, params: abi.ImuParameters, time_ns, readings, ranges, t0_ns, t1_ns) -> None:
        """Samples of the batch's IMU factors (in window order) for refresh_imu."""
        ll = C.POINTER(C.c_longlong)
        time_ns = np.ascontiguousarray(time_ns, dtype=np.int64)
        readings = np.ascontiguousarray(readings, dtype=np.float64)
        ranges = np.ascontiguousarray(ranges, dtype=np.int32)
        t0_ns = np.ascontiguousarray(t0_ns, dtype=np.int64)
        t1_ns = np.ascontiguousarray(t1_ns, dtype=np.int64)
        _check(lib().cgmli_solver_set_imu_samples(self._h, C.byref(params), time_ns.ctypes.data_as(ll), _p(readings), len(time_ns),
                                                  ranges.ctypes.data_as(abi.c_int_p), t0_ns.ctypes.data_as(ll),
                                                  t1_ns.ctypes.data_as(ll)), "cgmli_solver_set_imu_samples")

    def refresh_imu(self, gyro_threshold: float = 0.0003, accel_threshold: float = 0.02, wait: bool = True):
        """Re-preintegrates drifted IMU factors on the device; the count when wait."""
        n = C.c_int()
        _check(lib().cgmli_solver_refresh_imu(self._h, gyro_threshold, accel_threshold, C.byref(n) if wait else None),
               "cgmli_solver_refresh_imu")
        return n.value if wait else None

    def read_imu(self, w: int, count: int):
        out = (abi.FrozenImu * max(count, 1))()
        _check(lib().cgmli_solver_read_imu(self._h, w, out), "cgmli_solver_read_imu")
        return out

    def dims(self, w: int) -> tuple[int, int]:
        nr, nl = C.c_int(), C.c_int()
        _check(lib().cgmli_solver_window_dims(self._h, w, C.byref(nr), C.byref(nl)), "cgmli_solver_window_dims")
        return nr.value, nl.value

    def set_tuning(self, run_landmarks: int = 0, pair_chunk: int = 0, schur_rows: int = 0, lin_shape: int = 0,
                   trial_shape: int = 0, deterministic: int = 0) -> None:
        """Work decomposition and kernel shapes of the next set_windows (0: the default of each);
        deterministic=1 sums the J^T J and Schur passes in a fixed order (bitwise-reproducible
        windows, alone or in any batch)."""
        t = abi.Tuning(run_landmarks, pair_chunk, schur_rows, lin_shape, trial_shape, deterministic, 0.0)
        _check(lib().cgmli_solver_set_tuning(self._h, C.byref(t)), "cgmli_solver_set_tuning")

    def get_tuning(self) -> dict:
        t = abi.Tuning()
        _check(lib().cgmli_solver_get_tuning(self._h, C.byref(t)), "cgmli_solver_get_tuning")
        return dict(run_landmarks=t.run_landmarks, pair_chunk=t.pair_chunk, schur_rows=t.schur_rows, lin_shape=t.lin_shape,
                    trial_shape=t.trial_shape, deterministic=t.deterministic)

    def autotune(self, windows, iterations: int) -> dict:
        """Times candidate work decompositions on these windows, keeps the fastest
        and leaves the batch set with it."""
        arr = windows if isinstance(windows, C.Array) else _window_array(windows)
        t = abi.Tuning()
        _check(lib().cgmli_solver_autotune(self._h, arr, len(arr), iterations, C.byref(t)), "cgmli_solver_autotune")
        self._windows = arr
        self.count = len(arr)
        return dict(run_landmarks=t.run_landmarks, pair_chunk=t.pair_chunk, schur_rows=t.schur_rows, lin_shape=t.lin_shape,
                    trial_shape=t.trial_shape, deterministic=t.deterministic, ms=t.ms)

    def device_bytes(self) -> int:
        n = C.c_longlong()
        _check(lib().cgmli_solver_device_bytes(self._h, C.byref(n)), "cgmli_solver_device_bytes")
        return n.value

    def evaluate(self, derivatives: bool = True) -> None:
        """Per-factor residuals (and tangent Jacobians) of every window at its accepted states."""
        _check(lib().cgmli_solver_evaluate(self._h, int(derivatives)), "cgmli_solver_evaluate")

    def read_factors(self, w: int, jacobians: bool = True) -> dict:
        """Window w's factors in its observation order: residuals (F, 2), valid (F,), Jacobians (F, 2, 26)."""
        n = self._windows[w].num_observations
        r = np.zeros(2 * max(n, 1))
        v = np.zeros(max(n, 1), dtype=np.int32)
        J = np.zeros(abi.FACTOR_JACOBIAN * max(n, 1)) if jacobians else None
        _check(lib().cgmli_solver_read_factors(self._h, w, _p(r), v.ctypes.data_as(abi.c_int_p), _p(J) if J is not None else None),
               "cgmli_solver_read_factors")
        out = dict(residuals=r[:2 * n].reshape(n, 2), valid=v[:n].astype(bool))
        if J is not None:
            out["jacobians"] = J[:abi.FACTOR_JACOBIAN * n].reshape(n, 2, 26)
        return out

    def solve_host(self, iterations: int, fn, has_host=None) -> None:
        """LM solve with caller-evaluated factors.  fn(window, trial, poses (K,7), speed_bias (K,9),
        extrinsics (E,7), td) returns (H (Nr, Nr), g (Nr,), cost) at a linearization (trial False)
        and the cost alone at a trial (trial True); None fails the call."""
        dims = [self.dims(w)[0] for w in range(self.count)]
        wins = self._windows

        def cb(ctx, w, trial, poses, sb, ext, td, H, g, cost):
            try:
                K, E = wins[w].num_keyframes, wins[w].num_extrinsics
                P = np.ctypeslib.as_array(poses, shape=(K, 7)).copy()
                S = np.ctypeslib.as_array(sb, shape=(K, 9)).copy()
                X = np.ctypeslib.as_array(ext, shape=(E, 7)).copy()
                out = fn(w, bool(trial), P, S, X, float(td[0]))
                if out is None:
                    return 1
                if trial:
                    cost[0] = float(out)
                    return 0
                Hm, gv, c = out
                n = dims[w]
                np.ctypeslib.as_array(H, shape=(n * n,))[:] = np.asarray(Hm, dtype=np.float64).reshape(-1)
                np.ctypeslib.as_array(g, shape=(n,))[:] = np.asarray(gv, dtype=np.float64)
                cost[0] = float(c)
                return 0
            except Exception:  # noqa: BLE001 - reported to the library as a failed evaluation
                return 1

        cfn = abi.HOST_FACTOR_FN(cb)
        mask = None
        if has_host is not None:
            m = np.ascontiguousarray(has_host, dtype=np.uint8)
            mask = m.ctypes.data_as(C.POINTER(C.c_ubyte))
        _check(lib().cgmli_solver_solve_host(self._h, iterations, mask, cfn, None), "cgmli_solver_solve_host")

    def step(self, lam: float) -> None:
        _check(lib().cgmli_solver_step(self._h, lam), "cgmli_solver_step")

    def read_step(self, w: int) -> dict:
        nr, nl = self.dims(w)
        inc = np.zeros(nr + nl)
        cost, pred, trial = C.c_double(), C.c_double(), C.c_double()
        valid = C.c_int()
        code = lib().cgmli_solver_read_step(self._h, w, _p(inc), C.byref(cost), C.byref(pred), C.byref(trial), C.byref(valid))
        return dict(status=code, delta=inc, cost=cost.value, predicted=pred.value, trial_cost=trial.value,
                    trial_valid=bool(valid.value))

    def read_reduced(self, w: int):
        nr, _ = self.dims(w)
        S = np.zeros((nr, nr))
        rhs = np.zeros(nr)
        _check(lib().cgmli_solver_read_reduced(self._h, w, _p(S), _p(rhs)), "cgmli_solver_read_reduced")
        return S, rhs

    def checkpoint(self) -> None:
        _check(lib().cgmli_solver_checkpoint(self._h), "cgmli_solver_checkpoint")

    def rollback(self) -> None:
        _check(lib().cgmli_solver_rollback(self._h), "cgmli_solver_rollback")

    def kernel_times(self, enable: int = -1) -> dict:
        ms = np.zeros(len(abi.KERNEL_NAMES))
        calls = np.zeros(len(abi.KERNEL_NAMES), dtype=np.int32)
        _check(lib().cgmli_solver_kernel_times(self._h, enable, _p(ms), calls.ctypes.data_as(abi.c_int_p)),
               "cgmli_solver_kernel_times")
        return {n: (float(ms[i]), int(calls[i])) for i, n in enumerate(abi.KERNEL_NAMES)}

    def timing(self) -> tuple[float, int]:
        ms, n = C.c_double(), C.c_int()
        _check(lib().cgmli_solver_last_timing(self._h, C.byref(ms), C.byref(n)), "cgmli_solver_last_timing")
        return ms.value, n.value

    def marginalize(self, victims, policy: int = abi.MARGIN_OLD) -> None:
        """Schur marginalization of victims[w] (or -1 to skip) in every window."""
        v = np.ascontiguousarray(victims, dtype=np.int32)
        _check(lib().cgmli_solver_marginalize(self._h, v.ctypes.data_as(abi.c_int_p), policy), "cgmli_solver_marginalize")

    def read_prior(self, w: int) -> dict:
        """Square-root prior of window w: separator blocks, reference values, A (rank x cols), r0."""
        rank, cols, nb = C.c_int(), C.c_int(), C.c_int()
        code = lib().cgmli_solver_read_prior(self._h, w, C.byref(rank), C.byref(cols), C.byref(nb), None, None, None, None, None,
                                             None)
        if code != 0:
            return dict(status=code)
        k, m, b = rank.value, cols.value, nb.value
        kinds, idx = np.zeros(b, np.int32), np.zeros(b, np.int32)
        ref, A, r0, form = np.zeros(9 * b + 1), np.zeros(k * m), np.zeros(k), np.zeros(4)
        ip = abi.c_int_p
        code = lib().cgmli_solver_read_prior(self._h, w, C.byref(rank), C.byref(cols), C.byref(nb), kinds.ctypes.data_as(ip),
                                             idx.ctypes.data_as(ip), _p(ref), _p(A), _p(r0), _p(form))
        amb = int(sum(9 if t == abi.PRIOR_SPEED_BIAS else 1 if t == abi.PRIOR_TIME_OFFSET else 7 for t in kinds))
        return dict(status=code, rank=k, cols=m, kinds=kinds, index=idx, reference=ref[:amb], A=A.reshape(k, m), r0=r0,
                    robust_cost=form[0], rss=form[1], eliminated_reduction=form[2], cutoff=form[3])


def marg_eigen(H: np.ndarray):
    """Ascending eigenvalues and column eigenvectors of the symmetric H (lower triangle read)."""
    n = H.shape[0]
    Hc = np.asfortranarray(H, dtype=np.float64)
    ev, U = np.zeros(n), np.zeros((n, n), order="F")
    _check(lib().cgmli_marg_eigen(_p(Hc), n, _p(ev), _p(U)), "cgmli_marg_eigen")
    return ev, U


def marg_psd_solve(H: np.ndarray, rhs: np.ndarray, absolute_cutoff: float = 1e-12, relative_cutoff: float = 1e-9):
    n = H.shape[0]
    rhs2 = rhs.reshape(n, -1)
    Hc, Rc = np.asfortranarray(H, dtype=np.float64), np.asfortranarray(rhs2, dtype=np.float64)
    x = np.zeros(Rc.shape, order="F")
    _check(lib().cgmli_marg_psd_solve(_p(Hc), _p(Rc), n, Rc.shape[1], absolute_cutoff, relative_cutoff, _p(x)),
           "cgmli_marg_psd_solve")
    return x.reshape(rhs.shape)


def marg_subtract(coupling: np.ndarray, solution: np.ndarray, H: np.ndarray, g: np.ndarray):
    """[H | g] -= coupling^T solution, coupling nm x nr, solution nm x (nr + 1); returns new (H, g)."""
    nm, nr = coupling.shape
    Cc, Sc = np.asfortranarray(coupling, dtype=np.float64), np.asfortranarray(solution, dtype=np.float64)
    Ho, go = np.array(H, dtype=np.float64, order="F"), np.array(g, dtype=np.float64)
    _check(lib().cgmli_marg_subtract(_p(Cc), _p(Sc), nm, nr, _p(Ho), _p(go)), "cgmli_marg_subtract")
    return Ho, go


def imu_preintegrate(params: abi.ImuParameters, time_ns: np.ndarray, readings: np.ndarray, ranges: np.ndarray,
                     t0_ns: np.ndarray, t1_ns: np.ndarray, bias: np.ndarray):
    """Frozen IMU factors of len(t0_ns) intervals on the device (cgmli_imu_preintegrate).

    time_ns: int64 sample times; readings: (samples, 6) [gyro, accelerometer];
    ranges: (count, 2) sample index ranges [begin, end); bias: (count, 6) [b_g, b_a].
    Returns a ctypes array of abi.FrozenImu."""
    ll = C.POINTER(C.c_longlong)
    time_ns = np.ascontiguousarray(time_ns, dtype=np.int64)
    readings = np.ascontiguousarray(readings, dtype=np.float64)
    ranges = np.ascontiguousarray(ranges, dtype=np.int32)
    t0_ns = np.ascontiguousarray(t0_ns, dtype=np.int64)
    t1_ns = np.ascontiguousarray(t1_ns, dtype=np.int64)
    bias = np.ascontiguousarray(bias, dtype=np.float64)
    count = len(t0_ns)
    out = (abi.FrozenImu * max(count, 1))()
    _check(lib().cgmli_imu_preintegrate(C.byref(params), time_ns.ctypes.data_as(ll), _p(readings), len(time_ns),
                                        ranges.ctypes.data_as(abi.c_int_p), t0_ns.ctypes.data_as(ll), t1_ns.ctypes.data_as(ll),
                                        _p(bias), count, out), "cgmli_imu_preintegrate")
    return out


def imu_last_timing() -> float:
    """Kernel milliseconds of the last imu_preintegrate call."""
    ms = C.c_double()
    _check(lib().cgmli_imu_last_timing(C.byref(ms)), "cgmli_imu_last_timing")
    return ms.value


def _window_array(windows):
    arr = (abi.Window * len(windows))()
    for i, w in enumerate(windows):
        arr[i] = w.window if hasattr(w, "window") else w
    return arr


class Server:
    """Served mode: requests (one window each) are batched continuously on the
    device; see the cgmli_server_* functions of cgmli_backend.h.  The windows
    passed to submit() must stay alive until their request completes."""

    def __init__(self, device: int = 0, iterations: int = 1, policy: int = abi.MARGIN_OLD, max_batch_windows: int = 512,
                 memory_budget_bytes: int = 40 << 30, nis_threshold: float = 0.0, max_refits: int = 3, pre_gate: bool = False,
                 precision: int = abi.PRECISION_FP64, imu_params=None, imu_gyro_threshold: float = 3e-4,
                 imu_accel_threshold: float = 0.02, calibration_include_prior: bool = True, deterministic: bool = False):
        opt = abi.ServerOptions()
        opt.deterministic = int(deterministic)
        if imu_params is not None:
            opt.imu_params = imu_params
        opt.imu_gyro_threshold = imu_gyro_threshold
        opt.imu_accel_threshold = imu_accel_threshold
        opt.calibration_include_prior = int(calibration_include_prior)
        opt.device = device
        opt.max_batch_windows = max_batch_windows
        opt.memory_budget_bytes = memory_budget_bytes
        opt.iterations = iterations
        opt.policy = policy
        opt.nis_threshold = nis_threshold
        opt.max_refits = max_refits
        opt.pre_gate = int(pre_gate)
        opt.precision = precision
        self._h = C.c_void_p()
        _check(lib().cgmli_server_create(C.byref(opt), C.byref(self._h)), "cgmli_server_create")
        self._keep = {}

    def close(self):
        if self._h:
            lib().cgmli_server_destroy(self._h)
            self._h = C.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, window, victim: int = -1) -> int:
        """window: a synth.SynthWindow or an abi.Window; returns the ticket."""
        w = window.window if hasattr(window, "window") else window
        t = C.c_longlong()
        _check(lib().cgmli_server_submit(self._h, C.byref(w), victim, C.byref(t)), "cgmli_server_submit")
        self._keep[t.value] = window
        return t.value

    def submit_request(self, window, victim: int = -1, imu=None, calibration: bool = False) -> int:
        """A request with its optional parts: imu = (time_ns, readings, ranges, t0_ns, t1_ns)
        for the window's IMU factors (refreshed before the solve), calibration = the
        conditional calibration information at the solved states."""
        w = window.window if hasattr(window, "window") else window
        req = abi.ServerRequest()
        req.window = C.pointer(w)
        req.victim_kf = victim
        keep = [window, req]
        if imu is not None:
            t, rd, rg, t0, t1 = (np.ascontiguousarray(imu[0], np.int64), np.ascontiguousarray(imu[1], np.float64),
                                 np.ascontiguousarray(imu[2], np.int32), np.ascontiguousarray(imu[3], np.int64),
                                 np.ascontiguousarray(imu[4], np.int64))
            ll = C.POINTER(C.c_longlong)
            req.imu_sample_time_ns = t.ctypes.data_as(ll)
            req.imu_sample_readings = rd.ctypes.data_as(abi.c_double_p)
            req.num_imu_samples = len(t)
            req.imu_range = rg.ctypes.data_as(abi.c_int_p)
            req.imu_t0_ns = t0.ctypes.data_as(ll)
            req.imu_t1_ns = t1.ctypes.data_as(ll)
            keep += [t, rd, rg, t0, t1]
        req.calibration_information = int(calibration)
        tk = C.c_longlong()
        _check(lib().cgmli_server_submit_request(self._h, C.byref(req), C.byref(tk)), "cgmli_server_submit_request")
        self._keep[tk.value] = keep
        return tk.value

    def read_imu(self, ticket: int, count: int):
        """(factors after the refresh, how many were re-preintegrated)."""
        out = (abi.FrozenImu * max(count, 1))()
        n = C.c_int()
        _check(lib().cgmli_server_read_imu(self._h, ticket, out, C.byref(n)), "cgmli_server_read_imu")
        return list(out)[:count], n.value

    def read_merged_imu(self, ticket: int):
        """(outcome CGMLI_IMU_MERGE_*, merged factor or None) of a request marginalized
        with the IMU merge."""
        state = C.c_int()
        f = abi.FrozenImu()
        _check(lib().cgmli_server_read_merged_imu(self._h, ticket, C.byref(state), C.byref(f)), "cgmli_server_read_merged_imu")
        return state.value, (f if state.value == abi.IMU_MERGE_REINTEGRATED else None)

    def read_calibration_information(self, ticket: int) -> dict:
        size, nb = C.c_int(), C.c_int()
        code = lib().cgmli_server_read_calibration_information(self._h, ticket, C.byref(size), C.byref(nb), None, None, None, None)
        if code != 0:
            return dict(status=code)
        n, b = size.value, nb.value
        kinds, idx = np.zeros(b, np.int32), np.zeros(b, np.int32)
        cond, ev = np.zeros(n * n), np.zeros(n)
        _check(lib().cgmli_server_read_calibration_information(self._h, ticket, C.byref(size), C.byref(nb),
                                                               kinds.ctypes.data_as(abi.c_int_p), idx.ctypes.data_as(abi.c_int_p),
                                                               _p(cond), _p(ev)), "cgmli_server_read_calibration_information")
        return dict(status=0, size=n, kinds=kinds, index=idx, conditional=cond.reshape(n, n), eigenvalues=ev)

    def poll(self, ticket: int, wait: bool = True):
        """(report, latency_ms) once complete, None while pending (wait=False)."""
        rep, lat = abi.SolveReport(), C.c_double()
        code = lib().cgmli_server_poll(self._h, ticket, 1 if wait else 0, C.byref(rep), C.byref(lat))
        if code == abi.E_PENDING:
            return None
        _check(code, "cgmli_server_poll")
        return rep, lat.value

    def read_prior(self, ticket: int) -> dict:
        rank, cols, nb = C.c_int(), C.c_int(), C.c_int()
        code = lib().cgmli_server_read_prior(self._h, ticket, C.byref(rank), C.byref(cols), C.byref(nb), None, None, None, None,
                                             None)
        if code != 0:
            return dict(status=code)
        k, m, b = rank.value, cols.value, nb.value
        kinds, idx = np.zeros(b, np.int32), np.zeros(b, np.int32)
        ref, A, r0 = np.zeros(9 * b + 1), np.zeros(k * m), np.zeros(k)
        ip = abi.c_int_p
        code = lib().cgmli_server_read_prior(self._h, ticket, C.byref(rank), C.byref(cols), C.byref(nb), kinds.ctypes.data_as(ip),
                                             idx.ctypes.data_as(ip), _p(ref), _p(A), _p(r0))
        amb = int(sum(9 if t == abi.PRIOR_SPEED_BIAS else 1 if t == abi.PRIOR_TIME_OFFSET else 7 for t in kinds))
        return dict(status=code, rank=k, cols=m, kinds=kinds, index=idx, reference=ref[:amb], A=A.reshape(k, m), r0=r0)

    def device_bytes(self) -> int:
        """Device bytes both solvers of the server hold."""
        n = C.c_longlong()
        _check(lib().cgmli_server_device_bytes(self._h, C.byref(n)), "cgmli_server_device_bytes")
        return n.value

    def release(self, ticket: int) -> None:
        _check(lib().cgmli_server_release(self._h, ticket), "cgmli_server_release")
        self._keep.pop(ticket, None)

    def read_gate(self, ticket: int, num_observations: int):
        """(GateReport, rejected mask) of a completed gated request."""
        rep = abi.GateReport()
        mask = np.zeros(max(num_observations, 1), dtype=np.uint8)
        _check(lib().cgmli_server_read_gate(self._h, ticket, C.byref(rep), mask.ctypes.data_as(C.POINTER(C.c_ubyte))),
               "cgmli_server_read_gate")
        return rep, mask[:num_observations]

    def replay(self, windows, victims, arrival_s):
        """Replays a trace (window objects, victim per request, arrival times in s);
        returns (latency_ms array, status array, span_s)."""
        n = len(windows)
        ptrs = (C.POINTER(abi.Window) * n)(*[C.pointer(w.window if hasattr(w, "window") else w) for w in windows])
        vic = np.ascontiguousarray(victims, dtype=np.int32)
        arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
        lat, st, span = np.zeros(n), np.zeros(n, dtype=np.int32), C.c_double()
        _check(lib().cgmli_server_replay(self._h, ptrs, vic.ctypes.data_as(abi.c_int_p), _p(arr), n, _p(lat),
                                         st.ctypes.data_as(abi.c_int_p), C.byref(span)), "cgmli_server_replay")
        return lat, st, span.value

