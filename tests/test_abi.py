"""CPU checks of the C ABI library: it loads, exports every entry point that
include/cgmli_backend.h declares, its ctypes mirror matches the C layout, and
the generator is deterministic.  No compute is launched."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from cgmli_slam_b200 import abi, synth
from cgmli_slam_b200.build import INCLUDE, build_backend

HEADER = INCLUDE / "cgmli_backend.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cgmli_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(str(build_backend()))
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(abi.BACKEND_SYMBOLS) == names


def test_ctypes_layout_matches_c(tmp_path):
    src = tmp_path / "sizes.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   "int main(){printf(\"%zu %zu %zu %zu %zu %zu\\n\", sizeof(cgmli_window), sizeof(cgmli_frozen_imu),"
                   " sizeof(cgmli_solver_options), sizeof(cgmli_solve_report), offsetof(cgmli_window, prior_r0),"
                   " offsetof(cgmli_window, obs_P)); return 0;}\n")
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    assert got == [C.sizeof(abi.Window), C.sizeof(abi.FrozenImu), C.sizeof(abi.SolverOptions), C.sizeof(abi.SolveReport),
                   abi.Window.prior_r0.offset, abi.Window.obs_P.offset]


def test_ctypes_layout_of_server_options_and_tuning(tmp_path):
    src = tmp_path / "sizes2.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   "int main(){printf(\"%zu %zu %zu %zu\\n\", sizeof(cgmli_server_options), offsetof(cgmli_server_options, precision),"
                   " sizeof(cgmli_tuning), offsetof(cgmli_tuning, ms)); return 0;}\n")
    exe = tmp_path / "sizes2"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    assert got == [C.sizeof(abi.ServerOptions), abi.ServerOptions.precision.offset, C.sizeof(abi.Tuning), abi.Tuning.ms.offset]


def test_ctypes_layout_of_served_requests(tmp_path):
    """cgmli_server_request and the IMU / calibration tail of cgmli_server_options."""
    src = tmp_path / "sizes3.c"
    src.write_text(f'#include "{HEADER}"\n#include <stdio.h>\n#include <stddef.h>\n'
                   "int main(){printf(\"%zu %zu %zu %zu %zu %zu %zu\\n\", sizeof(cgmli_server_request),"
                   " offsetof(cgmli_server_request, num_imu_samples), offsetof(cgmli_server_request, calibration_information),"
                   " offsetof(cgmli_server_options, imu_params), offsetof(cgmli_server_options, imu_accel_threshold),"
                   " offsetof(cgmli_server_options, calibration_include_prior), offsetof(cgmli_server_options, deterministic));"
                   " return 0;}\n")
    exe = tmp_path / "sizes3"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    assert got == [C.sizeof(abi.ServerRequest), abi.ServerRequest.num_imu_samples.offset,
                   abi.ServerRequest.calibration_information.offset, abi.ServerOptions.imu_params.offset,
                   abi.ServerOptions.imu_accel_threshold.offset, abi.ServerOptions.calibration_include_prior.offset,
                   abi.ServerOptions.deterministic.offset]


def test_served_request_validation_without_gpu():
    """A negative refresh threshold is rejected when the server is created, before
    any device work."""
    lib = abi.declare_backend(C.CDLL(str(build_backend())))
    so = abi.ServerOptions()
    so.iterations, so.policy, so.max_refits = 1, abi.MARGIN_OLD, 3
    so.imu_gyro_threshold = -1.0
    srv = C.c_void_p()
    assert lib.cgmli_server_create(C.byref(so), C.byref(srv)) == abi.E_INVALID and not srv.value
    assert b"threshold" in lib.cgmli_last_error()


def test_server_deterministic_flag_is_validated_without_gpu():
    lib = abi.declare_backend(C.CDLL(str(build_backend())))
    so = abi.ServerOptions()
    so.iterations, so.policy, so.max_refits, so.deterministic = 1, abi.MARGIN_OLD, 3, 2
    srv = C.c_void_p()
    assert lib.cgmli_server_create(C.byref(so), C.byref(srv)) == abi.E_INVALID and not srv.value
    assert b"deterministic" in lib.cgmli_last_error()


def test_unknown_precision_is_rejected_before_any_device_work():
    """Options are validated first: an unknown precision is CGMLI_E_INVALID for the
    solver and the server alike, with or without a GPU."""
    lib = abi.declare_backend(C.CDLL(str(build_backend())))
    opt = abi.SolverOptions()
    lib.cgmli_default_options(C.byref(opt))
    opt.precision = 7
    h = C.c_void_p()
    assert lib.cgmli_solver_create(0, C.byref(opt), C.byref(h)) == abi.E_INVALID and not h.value
    assert b"precision" in lib.cgmli_last_error()
    so = abi.ServerOptions()
    so.iterations, so.policy, so.max_refits, so.precision = 1, abi.MARGIN_OLD, 3, 7
    srv = C.c_void_p()
    assert lib.cgmli_server_create(C.byref(so), C.byref(srv)) == abi.E_INVALID and not srv.value
    assert b"precision" in lib.cgmli_last_error()


def test_create_without_gpu_reports_an_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = abi.declare_backend(C.CDLL(str(build_backend())))
    h = C.c_void_p()
    code = lib.cgmli_solver_create(0, None, C.byref(h))
    assert code == 4 and not h.value
    assert b"device" in lib.cgmli_last_error()


def test_generator_is_deterministic():
    a = synth.SynthWindow(synth.C1, 123)
    b = synth.SynthWindow(synth.C1, 123)
    c = synth.SynthWindow(synth.C1, 124)
    assert np.array_equal(a.state_vector(), b.state_vector())
    assert a.F == b.F and not np.array_equal(a.state_vector()[:7], c.state_vector()[:7])


def test_generated_window_statistics():
    w = synth.SynthWindow(synth.C1, 5)
    rng = np.ctypeslib.as_array(w.window.lm_obs_begin, shape=(w.L + 1,))
    track = np.diff(rng) + 1  # + anchor observation
    assert w.L == 800 and track.min() >= 2 and track.max() <= 10
    out = w.outliers()
    assert 0.02 < out.mean() < 0.08
    assert w.window.num_imu == w.K - 1
