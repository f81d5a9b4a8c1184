"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference is quoted on Hilti 2023 robot replays, which are not available
here; these seeded windows stand in for them with the configured rig,
trajectory, landmark, noise, outlier and IMU statistics.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field, replace

import numpy as np

from . import abi
from .build import build_synth

_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        _LIB = abi.declare_synth(C.CDLL(str(build_synth())))
    return _LIB


@dataclass(frozen=True)
class WindowSpec:
    keyframes: int = 10
    landmarks: int = 800
    cameras: int = 4
    track_min: int = 2
    track_max: int = 10
    outlier_fraction: float = 0.05
    pixel_sigma: float = 1.0
    huber: float = 1.0
    with_imu: bool = True
    with_prior: bool = False
    estimate_extrinsics: bool = False
    per_camera_extrinsics: bool = False
    estimate_td: bool = False
    with_velocity: bool = False
    extrinsic_jitter_m: float = 0.0
    extrinsic_jitter_rad: float = 0.0
    init_position_sigma: float = 0.02
    init_rotation_sigma: float = math.radians(0.5)

    def params(self) -> abi.SynthParams:
        p = abi.SynthParams()
        for name, _ in abi.SynthParams._fields_:
            v = getattr(self, name)
            setattr(p, name, int(v) if isinstance(v, bool) else v)
        return p


# Benchmark configurations (sizes, noise, iterations) of the reference's
# headline measurement, numbered as listed there.
C1 = WindowSpec()  # plain single window, FP64, 1 LM iteration + OLD marginalization
C2 = WindowSpec(landmarks=3000, with_prior=True, estimate_extrinsics=True, per_camera_extrinsics=True,
                estimate_td=True, with_velocity=True)  # 24+1 calibration, 5 iterations, mixed precision
C3 = WindowSpec(keyframes=30, landmarks=20000, cameras=8, track_max=25, outlier_fraction=0.02,
                estimate_extrinsics=True, estimate_td=True, with_velocity=True)  # 10 iterations, SECOND_NEW
C4_BASE = WindowSpec(with_prior=True, estimate_extrinsics=True, per_camera_extrinsics=True, estimate_td=True,
                     with_velocity=True, extrinsic_jitter_m=0.01, extrinsic_jitter_rad=math.radians(0.3))
ITERATIONS = {"c1": 1, "c2": 5, "c3": 10, "c4": 5, "c5": 1}


def c4_spec(rng: np.random.Generator) -> WindowSpec:
    """One window of the batched configuration: K ~ U{6..15}, L ~ logU(200, 5000)."""
    k = int(rng.integers(6, 16))
    lm = int(round(math.exp(rng.uniform(math.log(200), math.log(5000)))))
    return replace(C4_BASE, keyframes=k, landmarks=lm)


class SynthWindow:
    """Owns one generated window; ``.window`` is the cgmli_window view."""

    def __init__(self, spec: WindowSpec, seed: int):
        self.spec = spec
        self.seed = seed
        params = spec.params()
        self._h = lib().cgmli_synth_make(C.byref(params), C.c_ulonglong(seed))
        if not self._h:
            raise RuntimeError("window generation failed")
        self.window = lib().cgmli_synth_window(self._h).contents

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.cgmli_synth_free(h)
            self._h = None

    # numpy views of the mutable state arrays
    def _view(self, ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,)) if n else np.zeros(0)

    @property
    def K(self):
        return self.window.num_keyframes

    @property
    def L(self):
        return self.window.num_landmarks

    @property
    def F(self):
        return self.window.num_observations

    def retained_dim(self) -> int:
        w = self.window
        return 15 * w.num_keyframes + (6 * w.num_extrinsics if w.estimate_extrinsics else 0) + (1 if (w.estimate_td and w.td) else 0)

    def poses(self):
        return self._view(self.window.poses, 7 * self.K)

    def speed_bias(self):
        return self._view(self.window.speed_bias, 9 * self.K)

    def extrinsics(self):
        return self._view(self.window.extrinsics, 7 * self.window.num_extrinsics)

    def rho(self):
        return self._view(self.window.rho, self.L)

    def td(self):
        return self._view(self.window.td, 1)

    def state_vector(self) -> np.ndarray:
        return np.concatenate([self.poses(), self.speed_bias(), self.extrinsics(), self.td(), self.rho()]).copy()

    def set_state_vector(self, x: np.ndarray) -> None:
        parts = [self.poses(), self.speed_bias(), self.extrinsics(), self.td(), self.rho()]
        off = 0
        for p in parts:
            p[:] = x[off:off + p.size]
            off += p.size

    def truth(self):
        K, E, L = self.K, self.window.num_extrinsics, self.L
        poses, sb, ext, rho, td = np.zeros(7 * K), np.zeros(9 * K), np.zeros(7 * E), np.zeros(L), np.zeros(1)
        dp = abi.c_double_p
        lib().cgmli_synth_truth(self._h, poses.ctypes.data_as(dp), sb.ctypes.data_as(dp), ext.ctypes.data_as(dp),
                                rho.ctypes.data_as(dp), td.ctypes.data_as(dp))
        return poses, sb, ext, rho, td

    def outliers(self) -> np.ndarray:
        out = np.zeros(self.F, dtype=np.int32)
        lib().cgmli_synth_outliers(self._h, out.ctypes.data_as(abi.c_int_p))
        return out


def make_windows(spec_or_name, count: int, seed: int = 0, threads: int | None = None) -> list[SynthWindow]:
    """``count`` windows with consecutive seeds; ``"c4"`` draws sizes per window.

    Generation runs on a thread pool (the C generator releases the GIL)."""
    if spec_or_name == "c4":
        rng = np.random.default_rng(seed)
        specs = [c4_spec(rng) for _ in range(count)]
    else:
        spec = {"c1": C1, "c2": C2, "c3": C3}.get(spec_or_name, spec_or_name)
        specs = [spec] * count
    lib()
    threads = threads or min(32, os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=threads) as pool:
        return list(pool.map(lambda i: SynthWindow(specs[i], seed + i), range(count)))


def window_array(windows: list[SynthWindow]):
    arr = (abi.Window * len(windows))()
    for i, w in enumerate(windows):
        arr[i] = w.window
    return arr
