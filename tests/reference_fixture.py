"""The reference's own geometry fixture, restated as cgmli_window inputs.

src/backend/tests/ManagedWindowRegression.cpp:28-66 builds a 2-camera rig
(camera 0: pinhole 640x480, f = 300, c = (320, 240), at the rig origin;
camera 1: EUCM 640x480, f = 120, c = (320, 240), alpha = 0.75, beta = 1, offset
0.2 m along x), four world points (0.3, 0.1, 4), (-0.4, 0.2, 5), (0.2, -0.3, 3)
and (1, 0, -0.2) (the last one behind camera 0, in the EUCM camera's rear
hemisphere), and keyframes 1, 2 with T_WB = (0.1 (id - 1), 0, 0), identity
rotation.  Keypoints are the points' projections stored as float, as the
fixture's cv::KeyPoint does; a camera stops listing keypoints at its first point
that does not project (so camera 0 sees points 0-2, camera 1 all four).

analyticSphereDerivativeAgreement (:168-234) evaluates the observations
{frame 1, camera 1, point 0} (same epoch as its anchor {1, 0, 0}),
{2, 1, 0} and {2, 1, 3} (anchored at {1, 1, 3}) in four scenarios:
0 as built; from 1 on, bearing velocities 0.15 (I - b b^T)(1, 2, -1) on the
anchor and the observation, reference time offsets 0.004 / -0.003, camera time
offset 0.001 (scenario 1) or 0.004, and the rig extrinsic
T((0.04, -0.02, 0.01), Exp(0.09, -0.06, 0.04)); from 2 on, keyframe 2 at
T((0.15, 0.02, -0.03), Exp(0.07, -0.03, 0.1)) and the inverse distance scaled by
0.6 (scenario 2) or 1.8 (scenario 3).  Its tolerances: residual 1e-8 (1 + |r|);
each Jacobian block against central differences in the left tangent with the
reference's steps (1e-6 translation, 1e-7 rotation and time offset,
min(0.01 rho, max(1e-12, 1e-6 rho)) for rho, WindowVisualFactor.cpp:584-601)
within 1e-7 + tol |numeric|, tol 1e-6 (1e-5 for the extrinsic and the time
offset; ModuleDebugArtifacts.hpp:41-58); same-epoch pose and shared-extrinsic
blocks exactly zero; rho = 0 rejected.

Observations are whitened as FrameStore::observation does
(src/backend/FrameStore.cpp:102-125) with sigma = 1 px (WindowDataTypes.hpp:16):
bearing = normalized back-projection, D = (I - b b^T) J / |ray|, covariance
sigma^2 (B^T D)(B^T D)^T with sphereBasis B (WindowVisualFactor.cpp:324-328),
P = L^-1 B^T.  This module is test infrastructure.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from cgmli_slam_b200 import abi

POINTS = np.array([[0.3, 0.1, 4.0], [-0.4, 0.2, 5.0], [0.2, -0.3, 3.0], [1.0, 0.0, -0.2]])
CAM_T = np.array([[0.0, 0.0, 0.0], [0.2, 0.0, 0.0]])  # T_SC translations (identity rotations)
PIXEL_SIGMA = 1.0
# (frame, camera, keypoint) of each observation and its landmark's anchor
OBSERVATIONS = [((1, 1, 0), (1, 0, 0)), ((2, 1, 0), (1, 0, 0)), ((2, 1, 3), (1, 1, 3))]


def exp_so3(theta):
    """Quaternion [x, y, z, w] of Exp(theta)."""
    theta = np.asarray(theta, dtype=np.float64)
    a = np.linalg.norm(theta)
    s = 0.5 - a * a / 48.0 if a < 1e-8 else math.sin(0.5 * a) / a
    return np.array([s * theta[0], s * theta[1], s * theta[2], math.cos(0.5 * a)])


def _pinhole_project(p):
    """PinholeCamera::project without distortion (None behind the camera or outside the image)."""
    if p[2] <= 0:
        return None
    u, v = 300.0 * p[0] / p[2] + 320.0, 300.0 * p[1] / p[2] + 240.0
    return (u, v) if 0 <= u < 640 and 0 <= v < 480 else None


def _pinhole_back(px):
    """Ray (x, y, 1) and its 3x2 pixel Jacobian (PinholeCamera.hpp:778-806)."""
    ray = np.array([(px[0] - 320.0) / 300.0, (px[1] - 240.0) / 300.0, 1.0])
    J = np.array([[1 / 300.0, 0.0], [0.0, 1 / 300.0], [0.0, 0.0]])
    return ray, J


_ALPHA, _BETA, _F, _C = 0.75, 1.0, 120.0, (320.0, 240.0)


def _eucm_project(p):
    """EucmCamera::project (EucmCamera.hpp:209-230)."""
    rho = math.sqrt(_BETA * (p[0] ** 2 + p[1] ** 2) + p[2] ** 2)
    rz = 1.0 / (_ALPHA * rho + (1.0 - _ALPHA) * p[2])
    u, v = _F * p[0] * rz + _C[0], _F * p[1] * rz + _C[1]
    return (u, v) if 0 <= u < 640 and 0 <= v < 480 else None


def _eucm_back(px):
    """Unit ray and its 3x2 pixel Jacobian (EucmCamera::backProject, EucmCamera.hpp:492-519)."""
    mx, my = (px[0] - _C[0]) / _F, (px[1] - _C[1]) / _F
    radius = mx * mx + my * my
    w = 1 - (2 * _ALPHA - 1) * _BETA * radius
    root = math.sqrt(w)
    den = _ALPHA * root + 1 - _ALPHA
    num = 1 - _BETA * _ALPHA * _ALPHA * radius
    ray = np.array([mx, my, num / den])
    unit = ray / np.linalg.norm(ray)
    dz = (-_BETA * _ALPHA * _ALPHA * den + num * _ALPHA * (2 * _ALPHA - 1) * _BETA / (2 * root)) / (den * den)
    deriv = np.array([[1 / _F, 0.0], [0.0, 1 / _F], [2 * mx * dz / _F, 2 * my * dz / _F]])
    J = (np.eye(3) - np.outer(unit, unit)) @ deriv / np.linalg.norm(ray)
    return unit, J


def keypoint(frame, camera, point):
    """Pixel of a world point in a frame's camera, stored as float (cv::KeyPoint)."""
    center = np.array([0.1 * (frame - 1), 0.0, 0.0]) + CAM_T[camera]
    pc = POINTS[point] - center
    px = _pinhole_project(pc) if camera == 0 else _eucm_project(pc)
    assert px is not None, "fixture point does not project"
    return np.float32(px[0]).astype(np.float64), np.float32(px[1]).astype(np.float64)


def sphere_basis(b):
    axis = np.array([1.0, 0.0, 0.0]) if abs(b[0]) < 0.8 else np.array([0.0, 1.0, 0.0])
    b0 = axis - b * b.dot(axis)
    b0 /= np.linalg.norm(b0)
    return np.stack([b0, np.cross(b, b0)], axis=1)


def observe(frame, camera, point, sigma=PIXEL_SIGMA):
    """Bearing and P = sqrtInfo B^T (2x3) of a keypoint (FrameStore::observation)."""
    px = keypoint(frame, camera, point)
    ray, J = _pinhole_back(px) if camera == 0 else _eucm_back(px)
    b = ray / np.linalg.norm(ray)
    D = (np.eye(3) - np.outer(b, b)) @ J / np.linalg.norm(ray)
    Bt = sphere_basis(b).T
    cov = sigma * sigma * (Bt @ D) @ (Bt @ D).T
    L = np.linalg.cholesky(cov)
    return b, np.linalg.solve(L, np.eye(2)) @ Bt


def bearing_velocity(b):
    return 0.15 * (np.eye(3) - np.outer(b, b)) @ np.array([1.0, 2.0, -1.0])


class FixtureWindow:
    """One window: keyframes 1 and 2, both cameras on one shared extrinsic (estimated),
    the camera time offset estimated, one landmark with one observation."""

    def __init__(self, observation, anchor, scenario, rho_scale=None):
        (fb, cb, kb), (fa, ca, ka) = observation, anchor
        assert kb == ka
        self.keep = []
        K, E, Cn, L, F = 2, 1, 2, 1, 1
        poses = np.zeros((K, 7))
        poses[:, 6] = 1.0
        poses[1, 0] = 0.1
        ext = np.array([[0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0]])
        td = np.array([0.0])
        ba, _ = observe(fa, ca, ka)
        bb, P = observe(fb, cb, kb)
        rho = 1.0 / np.linalg.norm(POINTS[ka] - (np.array([0.1 * (fa - 1), 0, 0]) + CAM_T[ca]))
        va, vb = np.zeros(3), np.zeros(3)
        ta, tb = 0.0, 0.0
        if scenario >= 1:
            va, vb = bearing_velocity(ba), bearing_velocity(bb)
            ta, tb = 0.004, -0.003
            td[0] = 0.001 if scenario == 1 else 0.004
            ext[0, :3] = [0.04, -0.02, 0.01]
            ext[0, 3:] = exp_so3([0.09, -0.06, 0.04])
        if scenario >= 2:
            poses[1, :3] = [0.15, 0.02, -0.03]
            poses[1, 3:] = exp_so3([0.07, -0.03, 0.1])
            rho *= 0.6 if scenario == 2 else 1.8
        if rho_scale is not None:
            rho *= rho_scale
        self.anchor_bearing = ba
        self.arrays = dict(
            poses=poses.ravel().copy(), sb=np.zeros(9 * K), ext=ext.ravel().copy(), td=td, rho=np.array([rho]),
            cam_R=np.tile(np.eye(3).ravel(), Cn), cam_t=CAM_T.ravel().copy(), cam_ext=np.zeros(Cn, np.int32),
            lm_kf=np.array([fa - 1], np.int32), lm_cam=np.array([ca], np.int32), lm_begin=np.array([0, F], np.int32),
            lm_bearing=ba.copy(), lm_vel=va.copy(), lm_time=np.array([ta]),
            obs_kf=np.array([fb - 1], np.int32), obs_cam=np.array([cb], np.int32), obs_bearing=bb.copy(),
            obs_P=P.ravel().copy(), obs_vel=vb.copy(), obs_time=np.array([tb]))
        a = self.arrays
        w = abi.Window()
        w.num_keyframes, w.num_cameras, w.num_extrinsics = K, Cn, E
        w.estimate_extrinsics, w.estimate_td = 1, 1
        w.num_landmarks, w.num_observations = L, F
        w.huber_scale, w.min_inverse_distance = 1.0, 1e-6
        dp, ip = abi.c_double_p, abi.c_int_p
        for name, key in (("poses", "poses"), ("speed_bias", "sb"), ("extrinsics", "ext"), ("td", "td"), ("rho", "rho"),
                          ("cam_R", "cam_R"), ("cam_t", "cam_t"), ("lm_anchor_bearing", "lm_bearing"),
                          ("lm_anchor_velocity", "lm_vel"), ("lm_anchor_time", "lm_time"), ("obs_bearing", "obs_bearing"),
                          ("obs_P", "obs_P"), ("obs_velocity", "obs_vel"), ("obs_time", "obs_time")):
            setattr(w, name, a[key].ctypes.data_as(dp))
        for name, key in (("cam_ext", "cam_ext"), ("lm_anchor_kf", "lm_kf"), ("lm_anchor_cam", "lm_cam"),
                          ("lm_obs_begin", "lm_begin"), ("obs_kf", "obs_kf"), ("obs_cam", "obs_cam")):
            setattr(w, name, a[key].ctypes.data_as(ip))
        self.window = w
        self.same_epoch = fa == fb
        self.a, self.b = fa - 1, fb - 1

    # tangent blocks of the factor, as the reference lists them: anchor pose,
    # observer pose (when another epoch), the shared extrinsic, td, rho
    def blocks(self):
        out = [("pose", self.a)]
        if self.b != self.a:
            out.append(("pose", self.b))
        return out + [("extrinsic", 0), ("td", 0), ("rho", 0)]

    @staticmethod
    def width(kind):
        return 6 if kind in ("pose", "extrinsic") else 1

    @staticmethod
    def step(kind, column, rho):
        """The reference's central-difference step (WindowVisualFactor.cpp:590-591)."""
        if kind in ("pose", "extrinsic"):
            return 1e-6 if column < 3 else 1e-7
        if kind == "rho":
            return min(0.01 * rho, max(1e-12, 1e-6 * rho))
        return 1e-7

    def analytic_block(self, J, kind, index):
        """The factor's analytic Jacobian over one block from the 2 x 26 layout."""
        if kind == "pose":
            blk = np.zeros((2, 6))
            if index == self.a:
                blk += J[:, 0:6]
            if index == self.b:
                blk += J[:, 6:12]
            return blk
        if kind == "extrinsic":
            return J[:, 12:18] + J[:, 18:24]
        return J[:, 24:25] if kind == "td" else J[:, 25:26]

    def perturbed(self, kind, index, column, h, plus):
        """A copy of this window with one tangent coordinate moved by +-h (left chart)."""
        from oracle import lib as olib  # the oracle's Plus is the chart's definition

        c = FixtureWindow.__new__(FixtureWindow)
        c.__dict__.update(self.__dict__)
        c.arrays = {k: v.copy() for k, v in self.arrays.items()}
        w = abi.Window()
        C.pointer(w)[0] = self.window
        c.window = w
        for name, key in (("poses", "poses"), ("extrinsics", "ext"), ("td", "td"), ("rho", "rho")):
            setattr(w, name, c.arrays[key].ctypes.data_as(abi.c_double_p))
        for name, key in (("speed_bias", "sb"), ("cam_R", "cam_R"), ("cam_t", "cam_t"), ("lm_anchor_bearing", "lm_bearing"),
                          ("lm_anchor_velocity", "lm_vel"), ("lm_anchor_time", "lm_time"), ("obs_bearing", "obs_bearing"),
                          ("obs_P", "obs_P"), ("obs_velocity", "obs_vel"), ("obs_time", "obs_time")):
            setattr(w, name, c.arrays[key].ctypes.data_as(abi.c_double_p))
        for name, key in (("cam_ext", "cam_ext"), ("lm_anchor_kf", "lm_kf"), ("lm_anchor_cam", "lm_cam"),
                          ("lm_obs_begin", "lm_begin"), ("obs_kf", "obs_kf"), ("obs_cam", "obs_cam")):
            setattr(w, name, c.arrays[key].ctypes.data_as(abi.c_int_p))
        s = h if plus else -h
        if kind in ("pose", "extrinsic"):
            arr = c.arrays["poses"] if kind == "pose" else c.arrays["ext"]
            x = arr[7 * index:7 * index + 7].copy()
            d = np.zeros(6)
            d[column] = s
            y = np.zeros(7)
            olib().oracle_pose_plus(x.ctypes.data_as(abi.c_double_p), d.ctypes.data_as(abi.c_double_p),
                                    y.ctypes.data_as(abi.c_double_p))
            arr[7 * index:7 * index + 7] = y
        elif kind == "td":
            c.arrays["td"][0] += s
        else:
            c.arrays["rho"][0] += s
        return c


def all_cases():
    """(observation, anchor, scenario) of analyticSphereDerivativeAgreement."""
    return [(o, a, s) for o, a in OBSERVATIONS for s in range(4)]
