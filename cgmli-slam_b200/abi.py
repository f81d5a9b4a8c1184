"""ctypes mirror of include/cgmli_backend.h and of the generator/oracle entry points."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent

c_double_p = C.POINTER(C.c_double)
c_int_p = C.POINTER(C.c_int)

OK = 0
ERRORS = {
    0: "ok", 1: "invalid input", 2: "non-finite", 3: "out of memory", 4: "CUDA error", 5: "not positive definite",
    6: "indefinite", 7: "unsupported", 8: "no acceptable step", 9: "size limit", 10: "cost mismatch",
    11: "pending",
}
PRECISION_FP64 = 0
PRECISION_MIXED = 1
PRIOR_POSE, PRIOR_SPEED_BIAS, PRIOR_EXTRINSIC, PRIOR_TIME_OFFSET = 0, 1, 2, 3
MARGIN_OLD, MARGIN_SECOND_NEW, MARGIN_SECOND_NEW_IMU_MERGE = 0, 1, 2
IMU_MERGE_NONE, IMU_MERGE_REINTEGRATED, IMU_MERGE_BRIDGE, IMU_MERGE_SUPPRESSED = 0, 1, 2, 3
MARG_EIGEN_NOALLOC_MAX_N = 256  # CGMLI_MARG_EIGEN_NOALLOC_MAX_N
FIX_POSE, FIX_VELOCITY, FIX_BIAS = 1, 2, 4
CHART_FULL, CHART_ROTATION_ONLY, CHART_FIXED = 0, 1, 2
FACTOR_JACOBIAN = 52  # CGMLI_FACTOR_JACOBIAN: 2 x 26 per factor
E_INVALID = 1
E_NONFINITE = 2
E_PENDING = 11


class FrozenImu(C.Structure):
    _fields_ = [
        ("duration", C.c_double), ("gravity", C.c_double),
        ("sensor_position", C.c_double * 3), ("sensor_quaternion", C.c_double * 4), ("gyros", C.c_double * 6),
        ("delta_quaternion", C.c_double * 4), ("delta_velocity", C.c_double * 3), ("delta_position", C.c_double * 3),
        ("reference_bias", C.c_double * 6),
        ("rotation_gyro", C.c_double * 9), ("velocity_gyro", C.c_double * 9), ("position_gyro", C.c_double * 9),
        ("velocity_accel", C.c_double * 9), ("position_accel", C.c_double * 9),
        ("whitening", C.c_double * 225),
    ]


class ImuParameters(C.Structure):
    _fields_ = [
        ("sigma_g_c", C.c_double), ("sigma_a_c", C.c_double), ("sigma_gw_c", C.c_double), ("sigma_aw_c", C.c_double),
        ("g_max", C.c_double), ("a_max", C.c_double), ("g", C.c_double), ("max_sample_gap", C.c_double),
        ("sensor_position", C.c_double * 3), ("sensor_quaternion", C.c_double * 4),
    ]


class Tuning(C.Structure):
    _fields_ = [("run_landmarks", C.c_int), ("pair_chunk", C.c_int), ("schur_rows", C.c_int), ("lin_shape", C.c_int),
                ("trial_shape", C.c_int), ("deterministic", C.c_int), ("ms", C.c_double)]


class GateReport(C.Structure):
    _fields_ = [("passes", C.c_int), ("rejected_pre", C.c_int), ("evaluated", C.c_int), ("rejected_last", C.c_int),
                ("rejected_total", C.c_int),
                ("nis_sum", C.c_double), ("nis_max", C.c_double)]


class Window(C.Structure):
    _fields_ = [
        ("num_keyframes", C.c_int), ("num_cameras", C.c_int), ("num_extrinsics", C.c_int),
        ("estimate_extrinsics", C.c_int), ("estimate_td", C.c_int), ("num_landmarks", C.c_int),
        ("num_observations", C.c_int), ("num_imu", C.c_int), ("prior_rank", C.c_int), ("prior_num_blocks", C.c_int),
        ("huber_scale", C.c_double), ("min_inverse_distance", C.c_double),
        ("poses", c_double_p), ("speed_bias", c_double_p), ("extrinsics", c_double_p), ("td", c_double_p), ("rho", c_double_p),
        ("cam_R", c_double_p), ("cam_t", c_double_p), ("cam_ext", c_int_p),
        ("lm_anchor_kf", c_int_p), ("lm_anchor_cam", c_int_p), ("lm_obs_begin", c_int_p),
        ("lm_anchor_bearing", c_double_p), ("lm_anchor_velocity", c_double_p), ("lm_anchor_time", c_double_p),
        ("obs_kf", c_int_p), ("obs_cam", c_int_p), ("obs_bearing", c_double_p), ("obs_P", c_double_p),
        ("obs_velocity", c_double_p), ("obs_time", c_double_p),
        ("imu", C.POINTER(FrozenImu)), ("imu_kf", c_int_p),
        ("prior_block_kind", c_int_p), ("prior_block_index", c_int_p),
        ("prior_ref", c_double_p), ("prior_A", c_double_p), ("prior_r0", c_double_p),
        ("kf_fixed", C.POINTER(C.c_ubyte)), ("ext_chart", C.POINTER(C.c_ubyte)), ("lm_fixed", C.POINTER(C.c_ubyte)),
    ]


class SolverOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("refinement_steps", C.c_int), ("initial_lambda", C.c_double),
                ("min_iterations", C.c_int), ("time_budget_s", C.c_double)]


class ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int), ("max_batch_windows", C.c_int), ("memory_budget_bytes", C.c_longlong),
                ("iterations", C.c_int), ("policy", C.c_int), ("nis_threshold", C.c_double), ("max_refits", C.c_int),
                ("pre_gate", C.c_int), ("precision", C.c_int), ("imu_params", ImuParameters),
                ("imu_gyro_threshold", C.c_double), ("imu_accel_threshold", C.c_double),
                ("calibration_include_prior", C.c_int), ("deterministic", C.c_int)]


class ServerRequest(C.Structure):
    _fields_ = [("window", C.POINTER(Window)), ("victim_kf", C.c_int), ("imu_sample_time_ns", C.POINTER(C.c_longlong)),
                ("imu_sample_readings", C.POINTER(C.c_double)), ("num_imu_samples", C.c_int), ("imu_range", C.POINTER(C.c_int)),
                ("imu_t0_ns", C.POINTER(C.c_longlong)), ("imu_t1_ns", C.POINTER(C.c_longlong)),
                ("calibration_information", C.c_int)]


class SolveReport(C.Structure):
    _fields_ = [("initial_cost", C.c_double), ("final_cost", C.c_double), ("lambda_", C.c_double),
                ("predicted_reduction", C.c_double), ("max_increment", C.c_double),
                ("iterations", C.c_int), ("accepted_steps", C.c_int), ("converged", C.c_int), ("status", C.c_int)]


class SynthParams(C.Structure):
    _fields_ = [
        ("keyframes", C.c_int), ("landmarks", C.c_int), ("cameras", C.c_int), ("track_min", C.c_int), ("track_max", C.c_int),
        ("outlier_fraction", C.c_double), ("pixel_sigma", C.c_double), ("huber", C.c_double),
        ("with_imu", C.c_int), ("with_prior", C.c_int), ("estimate_extrinsics", C.c_int),
        ("per_camera_extrinsics", C.c_int), ("estimate_td", C.c_int), ("with_velocity", C.c_int),
        ("extrinsic_jitter_m", C.c_double), ("extrinsic_jitter_rad", C.c_double),
        ("init_position_sigma", C.c_double), ("init_rotation_sigma", C.c_double),
    ]


# cgmli_host_factor_fn(ctx, window, trial, poses, speed_bias, extrinsics, td, H, g, cost)
HOST_FACTOR_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                             c_double_p, c_double_p)


def _proto(lib, name, restype, argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = argtypes
    return fn


def declare_backend(lib: C.CDLL) -> C.CDLL:
    W = C.POINTER(Window)
    S = C.c_void_p
    _proto(lib, "cgmli_last_error", C.c_char_p, [])
    _proto(lib, "cgmli_default_options", None, [C.POINTER(SolverOptions)])
    _proto(lib, "cgmli_topology_check", C.c_int, [W, C.c_int, C.c_int, c_double_p])
    _proto(lib, "cgmli_topology_check_tuned", C.c_int, [W, C.c_int, C.c_int, C.POINTER(Tuning), c_double_p])
    _proto(lib, "cgmli_topology_digest", C.c_int, [W, C.c_int, C.c_int, C.POINTER(Tuning), C.POINTER(C.c_ulonglong)])
    _proto(lib, "cgmli_solver_create", C.c_int, [C.c_int, C.POINTER(SolverOptions), C.POINTER(C.c_void_p)])
    _proto(lib, "cgmli_solver_destroy", None, [S])
    _proto(lib, "cgmli_solver_set_windows", C.c_int, [S, W, C.c_int])
    _proto(lib, "cgmli_solver_upload_states", C.c_int, [S, W, C.c_int])
    _proto(lib, "cgmli_solver_solve", C.c_int, [S, C.c_int])
    _proto(lib, "cgmli_solver_synchronize", C.c_int, [S])
    _proto(lib, "cgmli_solver_read_states", C.c_int, [S, W, C.c_int])
    _proto(lib, "cgmli_solver_read_reports", C.c_int, [S, C.POINTER(SolveReport), C.c_int])
    _proto(lib, "cgmli_solver_step", C.c_int, [S, C.c_double])
    _proto(lib, "cgmli_solver_read_step", C.c_int, [S, C.c_int, c_double_p, c_double_p, c_double_p, c_double_p, c_int_p])
    _proto(lib, "cgmli_solver_read_reduced", C.c_int, [S, C.c_int, c_double_p, c_double_p])
    _proto(lib, "cgmli_solver_window_dims", C.c_int, [S, C.c_int, c_int_p, c_int_p])
    _proto(lib, "cgmli_solver_last_timing", C.c_int, [S, c_double_p, c_int_p])
    _proto(lib, "cgmli_solver_marginalize", C.c_int, [S, c_int_p, C.c_int])
    _proto(lib, "cgmli_solver_read_prior", C.c_int,
           [S, C.c_int, c_int_p, c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p, c_double_p])
    _proto(lib, "cgmli_solver_checkpoint", C.c_int, [S])
    _proto(lib, "cgmli_solver_rollback", C.c_int, [S])
    _proto(lib, "cgmli_solver_kernel_times", C.c_int, [S, C.c_int, c_double_p, c_int_p])
    _proto(lib, "cgmli_marg_eigen", C.c_int, [c_double_p, C.c_int, c_double_p, c_double_p])
    _proto(lib, "cgmli_marg_psd_solve", C.c_int,
           [c_double_p, c_double_p, C.c_int, C.c_int, C.c_double, C.c_double, c_double_p])
    _proto(lib, "cgmli_marg_subtract", C.c_int, [c_double_p, c_double_p, C.c_int, C.c_int, c_double_p, c_double_p])
    _proto(lib, "cgmli_marg_eigen_noalloc", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p])
    V = C.c_void_p
    ll_p = C.POINTER(C.c_longlong)
    _proto(lib, "cgmli_server_create", C.c_int, [C.POINTER(ServerOptions), C.POINTER(C.c_void_p)])
    _proto(lib, "cgmli_server_destroy", None, [V])
    _proto(lib, "cgmli_server_submit", C.c_int, [V, W, C.c_int, ll_p])
    _proto(lib, "cgmli_server_submit_request", C.c_int, [V, C.POINTER(ServerRequest), ll_p])
    _proto(lib, "cgmli_server_read_imu", C.c_int, [V, C.c_longlong, C.POINTER(FrozenImu), c_int_p])
    _proto(lib, "cgmli_server_read_merged_imu", C.c_int, [V, C.c_longlong, c_int_p, C.POINTER(FrozenImu)])
    _proto(lib, "cgmli_server_read_calibration_information", C.c_int,
           [V, C.c_longlong, c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p])
    _proto(lib, "cgmli_server_poll", C.c_int, [V, C.c_longlong, C.c_int, C.POINTER(SolveReport), c_double_p])
    _proto(lib, "cgmli_server_read_prior", C.c_int,
           [V, C.c_longlong, c_int_p, c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p, c_double_p])
    _proto(lib, "cgmli_server_release", C.c_int, [V, C.c_longlong])
    _proto(lib, "cgmli_server_read_gate", C.c_int, [V, C.c_longlong, C.POINTER(GateReport), C.POINTER(C.c_ubyte)])
    _proto(lib, "cgmli_server_replay", C.c_int,
           [V, C.POINTER(W), c_int_p, c_double_p, C.c_int, c_double_p, c_int_p, c_double_p])
    _proto(lib, "cgmli_imu_preintegrate", C.c_int,
           [C.POINTER(ImuParameters), ll_p, c_double_p, C.c_int, c_int_p, ll_p, ll_p, c_double_p, C.c_int,
            C.POINTER(FrozenImu)])
    _proto(lib, "cgmli_imu_last_timing", C.c_int, [c_double_p])
    _proto(lib, "cgmli_solver_set_imu_samples", C.c_int,
           [S, C.POINTER(ImuParameters), ll_p, c_double_p, C.c_int, c_int_p, ll_p, ll_p])
    _proto(lib, "cgmli_solver_refresh_imu", C.c_int, [S, C.c_double, C.c_double, c_int_p])
    _proto(lib, "cgmli_solver_read_imu", C.c_int, [S, C.c_int, C.POINTER(FrozenImu)])
    _proto(lib, "cgmli_solver_solve_gated", C.c_int, [S, C.c_int, C.c_double, C.c_int, C.c_int])
    _proto(lib, "cgmli_solver_set_tuning", C.c_int, [S, C.POINTER(Tuning)])
    _proto(lib, "cgmli_solver_get_tuning", C.c_int, [S, C.POINTER(Tuning)])
    _proto(lib, "cgmli_solver_autotune", C.c_int, [S, W, C.c_int, C.c_int, C.POINTER(Tuning)])
    _proto(lib, "cgmli_solver_set_imu_merge_limits", C.c_int, [S, C.c_double, C.c_int])
    _proto(lib, "cgmli_solver_read_merged_imu", C.c_int, [S, C.c_int, c_int_p, C.POINTER(FrozenImu)])
    _proto(lib, "cgmli_solver_calibration_information", C.c_int, [S, C.c_int])
    _proto(lib, "cgmli_solver_read_calibration_information", C.c_int,
           [S, C.c_int, c_int_p, c_int_p, c_int_p, c_int_p, c_double_p, c_double_p])
    _proto(lib, "cgmli_solver_read_gate", C.c_int, [S, C.c_int, C.POINTER(GateReport), C.POINTER(C.c_ubyte)])
    _proto(lib, "cgmli_solver_device_bytes", C.c_int, [S, ll_p])
    _proto(lib, "cgmli_server_device_bytes", C.c_int, [V, ll_p])
    _proto(lib, "cgmli_solver_evaluate", C.c_int, [S, C.c_int])
    _proto(lib, "cgmli_solver_read_factors", C.c_int, [S, C.c_int, c_double_p, c_int_p, c_double_p])
    _proto(lib, "cgmli_solver_solve_host", C.c_int, [S, C.c_int, C.POINTER(C.c_ubyte), HOST_FACTOR_FN, C.c_void_p])
    return lib


def declare_synth(lib: C.CDLL) -> C.CDLL:
    _proto(lib, "cgmli_synth_make", C.c_void_p, [C.POINTER(SynthParams), C.c_ulonglong])
    _proto(lib, "cgmli_synth_free", None, [C.c_void_p])
    _proto(lib, "cgmli_synth_window", C.POINTER(Window), [C.c_void_p])
    _proto(lib, "cgmli_synth_truth", None, [C.c_void_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p])
    _proto(lib, "cgmli_synth_outliers", None, [C.c_void_p, c_int_p])
    return lib


# Every symbol include/cgmli_backend.h declares (checked by the CPU tests).
BACKEND_SYMBOLS = [
    "cgmli_last_error", "cgmli_default_options", "cgmli_solver_create", "cgmli_solver_destroy",
    "cgmli_solver_set_windows", "cgmli_solver_upload_states", "cgmli_solver_solve", "cgmli_solver_synchronize",
    "cgmli_solver_read_states", "cgmli_solver_read_reports", "cgmli_solver_step", "cgmli_solver_read_step",
    "cgmli_solver_read_reduced", "cgmli_solver_window_dims", "cgmli_solver_last_timing", "cgmli_solver_marginalize",
    "cgmli_solver_read_prior", "cgmli_marg_eigen", "cgmli_marg_psd_solve", "cgmli_marg_subtract",
    "cgmli_solver_checkpoint", "cgmli_solver_rollback", "cgmli_solver_kernel_times", "cgmli_topology_check",
    "cgmli_marg_eigen_noalloc", "cgmli_server_create", "cgmli_server_destroy", "cgmli_server_submit", "cgmli_server_poll",
    "cgmli_server_read_prior", "cgmli_server_release", "cgmli_server_replay", "cgmli_server_read_gate", "cgmli_imu_preintegrate",
    "cgmli_imu_last_timing", "cgmli_solver_set_imu_samples", "cgmli_solver_refresh_imu", "cgmli_solver_read_imu",
    "cgmli_solver_solve_gated", "cgmli_solver_read_gate", "cgmli_solver_set_imu_merge_limits", "cgmli_solver_read_merged_imu",
    "cgmli_solver_calibration_information", "cgmli_solver_read_calibration_information", "cgmli_topology_check_tuned", "cgmli_topology_digest",
    "cgmli_solver_set_tuning", "cgmli_solver_get_tuning", "cgmli_solver_autotune",
    "cgmli_solver_device_bytes", "cgmli_server_device_bytes", "cgmli_solver_evaluate", "cgmli_solver_read_factors",
    "cgmli_solver_solve_host", "cgmli_server_submit_request", "cgmli_server_read_imu", "cgmli_server_read_merged_imu", "cgmli_server_read_calibration_information",
]
KERNEL_NAMES = ["zero_acc", "linearize", "retained", "factor", "candidate", "backsub_trial", "retained_trial", "lm_update", "accept",
                "lin_pairs", "lin_schur"]
