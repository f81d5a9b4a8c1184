"""Windows and caller-evaluated factors shared by the boundary tests (test
infrastructure).

* charted(): a generated window with solve-time charts set, as the reference's
  optimizer sets them on its Ceres problem for one solve (constant blocks,
  BackendOptimizer.cpp:44-66; the bias-frozen speed/bias SubsetManifold and the
  rotation-only rig chart, :83-91,783-795).
* PriorAsHostFactor: the window's own square-root prior evaluated by the caller
  (r = r0 + A (x [-] x_ref), J = A D, from the oracle's prior factor), the form in
  which the reference hands a factor its device path does not take to
  solveOnline (retainedH = J^T J, retainedG = J^T r, BackendOptimizer.cpp:210-225).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from cgmli_slam_b200 import abi

U8 = C.POINTER(C.c_ubyte)


def set_charts(w, kf_fixed=None, ext_chart=None, lm_fixed=None):
    """Sets the chart arrays of SynthWindow w (kept alive on w)."""
    w._charts = []
    for name, values in (("kf_fixed", kf_fixed), ("ext_chart", ext_chart), ("lm_fixed", lm_fixed)):
        if values is None:
            setattr(w.window, name, U8())
            continue
        arr = np.ascontiguousarray(values, dtype=np.uint8)
        w._charts.append(arr)
        setattr(w.window, name, arr.ctypes.data_as(U8))
    return w


def retained_columns(win):
    """Retained column of each tangent entry of the window's prior, or -1."""
    K, E = win.num_keyframes, win.num_extrinsics
    est_ext, est_td = bool(win.estimate_extrinsics), bool(win.estimate_td and win.td)
    cols = []
    for b in range(win.prior_num_blocks):
        kind, idx = win.prior_block_kind[b], win.prior_block_index[b]
        if kind == abi.PRIOR_POSE:
            cols += [15 * idx + c for c in range(6)]
        elif kind == abi.PRIOR_SPEED_BIAS:
            cols += [15 * idx + 6 + c for c in range(9)]
        elif kind == abi.PRIOR_EXTRINSIC:
            cols += [15 * K + 6 * idx + c if est_ext else -1 for c in range(6)]
        else:
            cols += [15 * K + (6 * E if est_ext else 0) if est_td else -1]
    return np.array(cols)


class PriorAsHostFactor:
    """fn(window, trial, poses, speed_bias, extrinsics, td) of the host-factor API, evaluating
    the prior of `windows[window]` (the windows passed to the solver must carry no prior)."""

    def __init__(self, oracle, windows_with_prior, nr):
        self.O = oracle
        self.src = windows_with_prior
        self.nr = nr
        self.calls = [0, 0]

    def __call__(self, w, trial, poses, sb, ext, td):
        self.calls[int(trial)] += 1
        src = self.src[w]
        tmp = abi.Window()
        C.pointer(tmp)[0] = src
        keep = [np.ascontiguousarray(poses.ravel()), np.ascontiguousarray(sb.ravel()), np.ascontiguousarray(ext.ravel()),
                np.array([td])]
        tmp.poses, tmp.speed_bias, tmp.extrinsics = (k.ctypes.data_as(abi.c_double_p) for k in keep[:3])
        if src.td:
            tmp.td = keep[3].ctypes.data_as(abi.c_double_p)
        cols = retained_columns(src)
        rank = src.prior_rank
        r = np.zeros(rank)
        J = np.zeros(rank * len(cols))
        if not self.O.lib().oracle_prior_factor(C.byref(tmp), 0, r.ctypes.data_as(abi.c_double_p), J.ctypes.data_as(abi.c_double_p)):
            return None
        cost = 0.5 * float(r @ r)
        if trial:
            return cost
        Jr = np.zeros((rank, self.nr[w]))
        J = J.reshape(rank, len(cols))
        for j, c in enumerate(cols):
            if c >= 0:
                Jr[:, c] += J[:, j]
        return Jr.T @ Jr, Jr.T @ r, cost


def without_prior(win):
    """A copy of the window struct with its prior removed (same arrays otherwise)."""
    out = abi.Window()
    C.pointer(out)[0] = win
    out.prior_rank = 0
    out.prior_num_blocks = 0
    return out
