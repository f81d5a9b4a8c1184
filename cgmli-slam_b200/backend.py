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
                 initial_lambda: float = 1e-4, slabs_per_window: int = 0):
        opt = abi.SolverOptions()
        lib().cgmli_default_options(C.byref(opt))
        opt.precision = precision
        opt.refinement_steps = refinement
        opt.initial_lambda = initial_lambda
        opt.slabs_per_window = slabs_per_window
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

    def dims(self, w: int) -> tuple[int, int]:
        nr, nl = C.c_int(), C.c_int()
        _check(lib().cgmli_solver_window_dims(self._h, w, C.byref(nr), C.byref(nl)), "cgmli_solver_window_dims")
        return nr.value, nl.value

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


def _window_array(windows):
    arr = (abi.Window * len(windows))()
    for i, w in enumerate(windows):
        arr[i] = w.window if hasattr(w, "window") else w
    return arr
