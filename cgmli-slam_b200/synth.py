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


# ---- IMU streams for preintegration ------------------------------------------------
# Noise densities and saturation of the benchmark rig's IMU (sigma_g 1.7e-4,
# sigma_a 2e-3, random walks 2e-5 / 3e-3, 200 Hz).
IMU_DEFAULTS = dict(sigma_g_c=1.7e-4, sigma_a_c=2e-3, sigma_gw_c=2e-5, sigma_aw_c=3e-3, g_max=7.8, a_max=176.0, g=9.81,
                    max_sample_gap=0.05)


def imu_parameters(sensor_position=(0.0, 0.0, 0.0), sensor_quaternion=(0.0, 0.0, 0.0, 1.0), **overrides) -> abi.ImuParameters:
    p = abi.ImuParameters()
    for k, v in {**IMU_DEFAULTS, **overrides}.items():
        setattr(p, k, float(v))
    p.sensor_position[:] = list(sensor_position)
    p.sensor_quaternion[:] = list(sensor_quaternion)
    return p


@dataclass
class ImuStream:
    """Samples of one or more rigs and the keyframe intervals to preintegrate."""
    time_ns: np.ndarray   # (S,) int64, increasing within each rig
    readings: np.ndarray  # (S, 6) gyro, accelerometer
    ranges: np.ndarray    # (N, 2) sample range [begin, end) of each interval
    t0_ns: np.ndarray     # (N,) int64
    t1_ns: np.ndarray     # (N,) int64
    bias: np.ndarray      # (N, 6) linearization bias [b_g, b_a]

    @property
    def count(self) -> int:
        return len(self.t0_ns)


def imu_stream(rigs: int, keyframes: int, seed: int, rate: float = 200.0, spacing_s: float = 0.3,
               on_sample: bool = False) -> ImuStream:
    """Seeded IMU readings of ``rigs`` independent rigs, each with ``keyframes``
    keyframes ``spacing_s`` apart, and the keyframes-1 intervals of each rig.

    Readings follow a smooth random motion (gyro up to ~0.6 rad/s, specific
    force around gravity) with constant-plus-random-walk biases and white noise
    at the rig's densities.  Keyframe times fall between samples (the first and
    last step of every interval interpolate) unless ``on_sample``."""
    rng = np.random.default_rng(seed)
    h_ns = int(round(1e9 / rate))
    span = spacing_s * (keyframes - 1) + 0.1
    per_rig = int(np.ceil(span * rate)) + 4
    times, reads, ranges, t0s, t1s, biases = [], [], [], [], [], []
    offset = 0
    for rig in range(rigs):
        start_ns = int(1_000_000_000 * (1 + rig)) + int(rng.integers(0, h_ns))
        t_ns = start_ns + h_ns * np.arange(per_rig, dtype=np.int64)
        t = (t_ns - start_ns) * 1e-9
        freq = rng.uniform(0.5, 2.0, size=(2, 3))
        phase = rng.uniform(0, 2 * np.pi, size=(2, 3))
        amp_w = rng.uniform(0.1, 0.6, size=3)
        amp_a = rng.uniform(0.3, 2.0, size=3)
        bg = 2e-3 * rng.standard_normal(3) + np.cumsum(2e-5 * np.sqrt(1 / rate) * rng.standard_normal((per_rig, 3)), axis=0)
        ba = 2e-2 * rng.standard_normal(3) + np.cumsum(3e-3 * np.sqrt(1 / rate) * rng.standard_normal((per_rig, 3)), axis=0)
        gyro = amp_w * np.sin(freq[0] * t[:, None] * 2 * np.pi + phase[0]) + bg
        gyro += 1.7e-4 * np.sqrt(rate) * rng.standard_normal((per_rig, 3))
        acc = amp_a * np.sin(freq[1] * t[:, None] * 2 * np.pi + phase[1]) + np.array([0.0, 0.0, 9.81]) + ba
        acc += 2e-3 * np.sqrt(rate) * rng.standard_normal((per_rig, 3))
        times.append(t_ns)
        reads.append(np.hstack([gyro, acc]))
        kf = start_ns + int(0.05e9) + np.round(np.arange(keyframes) * spacing_s * 1e9).astype(np.int64)
        if on_sample:
            kf = start_ns + h_ns * np.round((kf - start_ns) / h_ns).astype(np.int64)
        else:
            kf = kf + rng.integers(1, h_ns - 1, size=keyframes)
        for k in range(keyframes - 1):
            a, b = int(kf[k]), int(kf[k + 1])
            lo = max(int(np.searchsorted(t_ns, a, side="right")) - 2, 0)
            hi = min(int(np.searchsorted(t_ns, b, side="left")) + 2, per_rig)
            ranges.append((offset + lo, offset + hi))
            t0s.append(a)
            t1s.append(b)
            i = int(np.searchsorted(t_ns, a))
            biases.append(np.concatenate([bg[i], ba[i]]) + np.concatenate([1e-4 * rng.standard_normal(3),
                                                                            5e-3 * rng.standard_normal(3)]))
        offset += per_rig
    return ImuStream(np.concatenate(times), np.vstack(reads), np.array(ranges, dtype=np.int32), np.array(t0s, dtype=np.int64),
                     np.array(t1s, dtype=np.int64), np.array(biases))


# ---- sliding-window sequences (configuration 2's chained prior) -----------------
class SubWindow:
    """Keyframes [start, start + K) of a long generated window, as a sliding
    window holds them after `start` OLD marginalizations: landmarks with an
    observation (or anchor) on an earlier keyframe were eliminated with it
    (the OLD elimination set, SlidingWindowManager.cpp:627-652); a landmark's
    observations beyond the window's last keyframe are not made yet.  States
    are copied from the long window (its current estimates); the prior is set
    by set_prior from the previous window's marginalization."""

    def __init__(self, long: "SynthWindow", start: int, K: int):
        src = long.window
        Kt = src.num_keyframes
        assert 0 <= start and start + K <= Kt
        self.long, self.start, self.K = long, start, K
        E, Cn = src.num_extrinsics, src.num_cameras
        Lt = src.num_landmarks
        begin = np.ctypeslib.as_array(src.lm_obs_begin, shape=(Lt + 1,))
        Ft = int(begin[-1])
        lm_kf = np.ctypeslib.as_array(src.lm_anchor_kf, shape=(Lt,))
        obs_kf = np.ctypeslib.as_array(src.obs_kf, shape=(Ft,))
        lms, obs, new_begin = [], [], [0]
        for l in range(Lt):
            a = int(lm_kf[l])
            ks = obs_kf[begin[l]:begin[l + 1]]
            if a < start or a >= start + K or np.any(ks < start):
                continue
            keep = [f for f in range(begin[l], begin[l + 1]) if obs_kf[f] < start + K]
            if not keep:
                continue
            lms.append(l)
            obs.extend(keep)
            new_begin.append(len(obs))
        self.lms = np.array(lms, dtype=np.int64)
        self.obs = np.array(obs, dtype=np.int64)

        def arr(ptr, n, dtype=np.float64):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy() if ptr else None

        L, F = len(lms), len(obs)
        kf = slice(start, start + K)
        a = {}
        a["poses"] = long.poses().reshape(Kt, 7)[kf].ravel().copy()
        a["sb"] = long.speed_bias().reshape(Kt, 9)[kf].ravel().copy()
        a["ext"] = long.extrinsics().copy()
        a["td"] = long.td().copy()
        a["rho"] = long.rho()[self.lms].copy()
        a["cam_R"], a["cam_t"] = arr(src.cam_R, 9 * Cn), arr(src.cam_t, 3 * Cn)
        a["cam_ext"] = arr(src.cam_ext, Cn, np.int32)
        a["lm_kf"] = (lm_kf[self.lms] - start).astype(np.int32)
        a["lm_cam"] = np.ctypeslib.as_array(src.lm_anchor_cam, shape=(Lt,))[self.lms].astype(np.int32).copy()
        a["lm_begin"] = np.array(new_begin, dtype=np.int32)
        a["lm_bearing"] = np.ctypeslib.as_array(src.lm_anchor_bearing, shape=(Lt, 3))[self.lms].ravel().copy()
        a["obs_kf"] = (obs_kf[self.obs] - start).astype(np.int32)
        a["obs_cam"] = np.ctypeslib.as_array(src.obs_cam, shape=(Ft,))[self.obs].astype(np.int32).copy()
        a["obs_bearing"] = np.ctypeslib.as_array(src.obs_bearing, shape=(Ft, 3))[self.obs].ravel().copy()
        a["obs_P"] = np.ctypeslib.as_array(src.obs_P, shape=(Ft, 6))[self.obs].ravel().copy()
        if src.lm_anchor_velocity:
            a["lm_vel"] = np.ctypeslib.as_array(src.lm_anchor_velocity, shape=(Lt, 3))[self.lms].ravel().copy()
        if src.obs_velocity:
            a["obs_vel"] = np.ctypeslib.as_array(src.obs_velocity, shape=(Ft, 3))[self.obs].ravel().copy()
        imu_kf = np.ctypeslib.as_array(src.imu_kf, shape=(src.num_imu,)) if src.num_imu else np.zeros(0, np.int32)
        sel = [i for i in range(src.num_imu) if start <= imu_kf[i] and imu_kf[i] + 1 < start + K]
        self.imu = (abi.FrozenImu * max(len(sel), 1))()
        for j, i in enumerate(sel):
            self.imu[j] = src.imu[i]
        a["imu_kf"] = (imu_kf[sel] - start).astype(np.int32) if sel else np.zeros(1, np.int32)
        self.arrays = a
        w = abi.Window()
        w.num_keyframes, w.num_cameras, w.num_extrinsics = K, Cn, E
        w.estimate_extrinsics, w.estimate_td = src.estimate_extrinsics, src.estimate_td
        w.num_landmarks, w.num_observations, w.num_imu = L, F, len(sel)
        w.huber_scale, w.min_inverse_distance = src.huber_scale, src.min_inverse_distance
        dp, ip = abi.c_double_p, abi.c_int_p
        for name, key in (("poses", "poses"), ("speed_bias", "sb"), ("extrinsics", "ext"), ("td", "td"), ("rho", "rho"),
                          ("cam_R", "cam_R"), ("cam_t", "cam_t"), ("lm_anchor_bearing", "lm_bearing"),
                          ("obs_bearing", "obs_bearing"), ("obs_P", "obs_P")):
            setattr(w, name, a[key].ctypes.data_as(dp))
        for name, key in (("lm_anchor_velocity", "lm_vel"), ("obs_velocity", "obs_vel")):
            if key in a:
                setattr(w, name, a[key].ctypes.data_as(dp))
        for name, key in (("cam_ext", "cam_ext"), ("lm_anchor_kf", "lm_kf"), ("lm_anchor_cam", "lm_cam"),
                          ("lm_obs_begin", "lm_begin"), ("obs_kf", "obs_kf"), ("obs_cam", "obs_cam"), ("imu_kf", "imu_kf")):
            setattr(w, name, a[key].ctypes.data_as(ip))
        if sel:
            w.imu = self.imu
        self.window = w

    @property
    def L(self):
        return self.window.num_landmarks

    def retained_dim(self) -> int:
        w = self.window
        return 15 * w.num_keyframes + (6 * w.num_extrinsics if w.estimate_extrinsics else 0) + (1 if (w.estimate_td and w.td) else 0)

    def set_prior(self, prior: dict, shift: int) -> None:
        """The square-root prior of the previous window's marginalization (read_prior), its
        keyframe blocks moved down by `shift` (the keyframes that left the window)."""
        kinds = np.ascontiguousarray(prior["kinds"], dtype=np.int32)
        idx = np.array([i - shift if k in (abi.PRIOR_POSE, abi.PRIOR_SPEED_BIAS) else i for k, i in zip(kinds, prior["index"])],
                       dtype=np.int32)
        assert np.all(idx >= 0)
        amb = int(sum(9 if k == abi.PRIOR_SPEED_BIAS else 1 if k == abi.PRIOR_TIME_OFFSET else 7 for k in kinds))
        self.prior = dict(kinds=kinds, index=idx, ref=np.ascontiguousarray(prior["reference"][:amb]),
                          A=np.ascontiguousarray(prior["A"]).ravel().copy(), r0=np.ascontiguousarray(prior["r0"]).copy())
        w, p = self.window, self.prior
        w.prior_rank, w.prior_num_blocks = int(prior["rank"]), len(kinds)
        w.prior_block_kind, w.prior_block_index = p["kinds"].ctypes.data_as(abi.c_int_p), p["index"].ctypes.data_as(abi.c_int_p)
        w.prior_ref, w.prior_A, w.prior_r0 = (p[k].ctypes.data_as(abi.c_double_p) for k in ("ref", "A", "r0"))

    def store(self) -> None:
        """Writes this window's states back into the long window (the next window starts from them)."""
        Kt = self.long.window.num_keyframes
        kf = slice(self.start, self.start + self.K)
        self.long.poses().reshape(Kt, 7)[kf] = self.arrays["poses"].reshape(self.K, 7)
        self.long.speed_bias().reshape(Kt, 9)[kf] = self.arrays["sb"].reshape(self.K, 9)
        self.long.extrinsics()[:] = self.arrays["ext"]
        self.long.td()[:] = self.arrays["td"]
        self.long.rho()[self.lms] = self.arrays["rho"]

    def state_vector(self) -> np.ndarray:
        a = self.arrays
        return np.concatenate([a["poses"], a["sb"], a["ext"], a["td"], a["rho"]]).copy()

    def set_state_vector(self, x: np.ndarray) -> None:
        off = 0
        for k in ("poses", "sb", "ext", "td", "rho"):
            n = self.arrays[k].size
            self.arrays[k][:] = x[off:off + n]
            off += n


# Configuration 2 as a sequence: 15 keyframes generated at once, sliding windows of 10; the
# fifth window's prior comes from five chained OLD marginalizations of the ones before it.
C2_CHAIN_KEYFRAMES = 15
C2_CHAIN_LANDMARKS = 6000


def c2_long_window(seed: int, landmarks: int = C2_CHAIN_LANDMARKS) -> "SynthWindow":
    return SynthWindow(replace(C2, keyframes=C2_CHAIN_KEYFRAMES, landmarks=landmarks, with_prior=False), seed)
