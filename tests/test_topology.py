"""Host-side batch layout on CPU (no GPU): cgmli_topology_check builds the
device layout of a batch of windows and verifies its invariants - landmark
order is a permutation, observation ranges and keyframe/extrinsic slots match
the caller's data, the key order of the J^T J pass is sorted, and every work
unit (runs of tiles, pair chunks, Schur chunks) stays inside its window and
covers each landmark / observation exactly once."""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import pytest

from cgmli_slam_b200 import abi, synth
from cgmli_slam_b200.build import build_backend


@pytest.fixture(scope="module")
def lib():
    return abi.declare_backend(C.CDLL(str(build_backend())))


def check(lib, windows, threads=0):
    arr = synth.window_array(windows)
    sec = C.c_double()
    code = lib.cgmli_topology_check(arr, len(arr), threads, C.byref(sec))
    return code, sec.value, lib.cgmli_last_error().decode()


SPECS = {
    "c1": synth.C1,
    "c2": synth.C2,
    "shared_calib_td": replace(synth.C1, landmarks=400, estimate_extrinsics=True, estimate_td=True, with_velocity=True,
                               with_prior=True),
    "no_imu": replace(synth.C1, keyframes=6, landmarks=300, with_imu=False),
    "imu_only": replace(synth.C1, keyframes=5, landmarks=0, with_prior=True),
    "long_tracks_8cam": replace(synth.C3, keyframes=12, landmarks=1500),
}


@pytest.mark.parametrize("name", list(SPECS))
def test_single_window_layout(lib, name):
    code, _, why = check(lib, [synth.SynthWindow(SPECS[name], 3)])
    assert code == 0, why


@pytest.mark.parametrize("threads", [1, 4, 0])
def test_batched_layout_any_thread_count(lib, threads):
    windows = synth.make_windows("c4", 24, seed=5)
    code, sec, why = check(lib, windows, threads)
    assert code == 0, why
    assert sec > 0


def test_large_window_layout(lib):
    code, _, why = check(lib, [synth.SynthWindow(replace(synth.C3, landmarks=6000), 2)])
    assert code == 0, why


def test_malformed_window_is_rejected(lib):
    w = synth.SynthWindow(replace(synth.C1, keyframes=4, landmarks=60), 9)
    arr = synth.window_array([w])
    arr[0].num_keyframes = 2  # observations now reference missing keyframes
    code = lib.cgmli_topology_check(arr, 1, 0, None)
    assert code == 1
    assert b"window 0" in lib.cgmli_last_error()


def test_window_above_visual_limit_is_rejected(lib):
    w = synth.SynthWindow(replace(synth.C1, keyframes=4, landmarks=60), 9)
    arr = synth.window_array([w])
    arr[0].num_extrinsics = 80  # 6K + 6E + 1 > 400 with per-camera extrinsics estimated
    arr[0].estimate_extrinsics = 1
    code = lib.cgmli_topology_check(arr, 1, 0, None)
    assert code == 9  # CGMLI_E_LIMIT


@pytest.mark.parametrize("tuning", [(2, 8, 8, 0, 0, 0), (8, 64, 32, 1, 2, 0), (64, 1024, 128, 3, 1, 0), (0, 0, 0, 2, 0, 0),
                                    (4096, 128, 16, 0, 0, 0), (0, 0, 0, 0, 0, 1), (2, 8, 8, 0, 0, 1), (64, 1024, 128, 3, 1, 1)])
def test_tuned_layout(lib, tuning):
    """Every work decomposition the autotuner may pick keeps the invariants
    (runs cover each landmark once, pair chunks and Schur chunks within their
    limits and windows; in deterministic mode the units tile each window's chunks
    in slot order and the slots fill the slot array)."""
    windows = synth.make_windows("c4", 12, seed=17)
    arr = synth.window_array(windows)
    t = abi.Tuning(*tuning, 0.0)
    code = lib.cgmli_topology_check_tuned(arr, len(arr), 0, C.byref(t), None)
    assert code == 0, lib.cgmli_last_error().decode()


@pytest.mark.parametrize("tuning", [(-1, 32, 128, 0, 0, 0), (0, 4, 128, 0, 0, 0), (0, 2048, 128, 0, 0, 0), (0, 32, 4, 0, 0, 0),
                                    (0, 32, 256, 0, 0, 0), (0, 32, 128, 4, 0, 0), (0, 32, 128, 0, 3, 0), (0, 32, 128, -1, 0, 0),
                                    (0, 32, 128, 0, 0, 2), (0, 32, 128, 0, 0, -1)])
def test_tuning_outside_its_ranges_is_rejected(lib, tuning):
    windows = synth.make_windows("c4", 2, seed=3)
    arr = synth.window_array(windows)
    t = abi.Tuning(*tuning, 0.0)
    assert lib.cgmli_topology_check_tuned(arr, len(arr), 0, C.byref(t), None) == abi.E_INVALID


def _digest(lib, windows, threads, tuning=None):
    arr = synth.window_array(windows)
    out = C.c_ulonglong()
    code = lib.cgmli_topology_digest(arr, len(arr), threads, C.byref(tuning) if tuning else None, C.byref(out))
    assert code == 0, lib.cgmli_last_error().decode()
    return out.value


def test_layout_is_the_same_for_any_thread_count(lib):
    """A batch with a window of several thousand landmarks and few windows is built in
    range steps split over the threads; a batch of many windows is built window by
    window, largest first.  Either way the layout (the digest of every uploaded array)
    does not depend on the thread count, and every such build keeps the invariants."""
    big = [synth.SynthWindow(replace(synth.C3, keyframes=14, landmarks=3000), 4),
           synth.SynthWindow(replace(synth.C1, landmarks=300), 5)]
    many = synth.make_windows("c4", 20, seed=23)
    for windows in (big, many):
        digests = {_digest(lib, windows, t) for t in (1, 2, 3, 8)}
        assert len(digests) == 1
        for t in (1, 3):
            code, _, why = check(lib, windows, t)
            assert code == 0, why


def test_layout_digest_sees_the_decomposition(lib):
    windows = synth.make_windows("c4", 6, seed=29)
    a = _digest(lib, windows, 2, abi.Tuning(8, 32, 128, 0, 0, 0, 0.0))
    b = _digest(lib, windows, 2, abi.Tuning(16, 32, 128, 0, 0, 0, 0.0))
    c = _digest(lib, windows, 2, abi.Tuning(8, 32, 128, 0, 0, 1, 0.0))
    assert len({a, b, c}) == 3


def test_deterministic_units_follow_the_window_alone(lib):
    """Deterministic mode splits each window's pair and Schur chunks into units by the
    window alone (in chunk order, at most 128 of each): the layout is the same for any
    thread count (range steps or whole windows) and keeps the unit invariants."""
    det = abi.Tuning(0, 32, 128, 0, 0, 1, 0.0)
    big = [synth.SynthWindow(replace(synth.C3, keyframes=14, landmarks=3000), 4),
           synth.SynthWindow(replace(synth.C1, landmarks=300), 5)]
    many = synth.make_windows("c4", 20, seed=23)
    for windows in (big, many):
        assert len({_digest(lib, windows, t, det) for t in (1, 2, 3, 8)}) == 1
        arr = synth.window_array(windows)
        assert lib.cgmli_topology_check_tuned(arr, len(arr), 3, C.byref(det), None) == 0, lib.cgmli_last_error().decode()
