"""CPU tests of the oracle's SECOND_NEW IMU merge (SlidingWindowManager::
prepareEviction, src/backend/SlidingWindowManager.cpp:263-310; mergeBodyImuRecords,
src/factor/BodyImuFactor.cpp:306-388)."""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from cgmli_slam_b200 import abi, synth

SPEC = replace(synth.C1, keyframes=6, landmarks=300)


def stream_window(oracle, seed, spec=SPEC):
    w = synth.SynthWindow(spec, seed)
    K, nimu = w.K, w.window.num_imu
    kf = np.array([w.window.imu_kf[q] for q in range(nimu)])
    s = synth.imu_stream(1, K, seed + 1)
    prm = synth.imu_parameters()
    sb = w.speed_bias().reshape(K, 9)
    args = (s.time_ns, s.readings, s.ranges[kf], s.t0_ns[kf], s.t1_ns[kf])
    st, built = oracle.imu_preintegrate(prm, *args, sb[kf, 3:9])
    assert st == 0
    for q in range(nimu):
        w.window.imu[q] = built[q]
    return w, prm, args


def test_merged_factor_is_the_concatenated_interval(oracle):
    """The merged factor is the preintegration of both edges' samples from the
    left edge's start to the right edge's end at the left keyframe's bias."""
    w, prm, (t, rd, rg, t0, t1) = stream_window(oracle, 61)
    v = w.K - 2
    r = oracle.marginalize_window_merge(w.window, v, prm, t, rd, rg, t0, t1)
    assert r["status"] == 0 and r["merge"] == abi.IMU_MERGE_REINTEGRATED
    left, right = v - 1, v
    sb = w.speed_bias().reshape(w.K, 9)
    st, direct = oracle.imu_preintegrate(prm, t, rd, [[rg[left][0], rg[right][1]]], [t0[left]], [t1[right]], sb[None, v - 1, 3:9])
    assert st == 0 and bytes(direct[0]) == bytes(r["merged"])
    assert abs(r["merged"].duration - (t1[right] - t0[left]) * 1e-9) < 1e-15


def test_merged_edges_leave_the_separator(oracle):
    """With the merge the victim's IMU edges do not enter the Schur step: the
    neighbours' speed/bias blocks leave the separator (no other factor there);
    with the bridge (plain SECOND_NEW) they are in it."""
    w, prm, args = stream_window(oracle, 62)
    v = w.K - 2
    merge = oracle.marginalize_window_merge(w.window, v, prm, *args)
    bridge = oracle.marginalize_window(w.window, v, abi.MARGIN_SECOND_NEW)
    sb_blocks = lambda r: {int(i) for k, i in zip(r["kinds"], r["index"]) if k == abi.PRIOR_SPEED_BIAS}
    assert {v - 1, v + 1} <= sb_blocks(bridge)
    assert not ({v - 1, v + 1} & sb_blocks(merge))
    assert merge["rank"] < bridge["rank"]


def test_suppressed_and_bridge_conditions(oracle):
    w, prm, args = stream_window(oracle, 63)
    v = w.K - 2
    # longer than the maximum duration: both edges dropped, no factor
    r = oracle.marginalize_window_merge(w.window, v, prm, *args, max_interval=0.5)
    assert r["status"] == 0 and r["merge"] == abi.IMU_MERGE_SUPPRESSED and r["merged"] is None
    # the sample budget
    r = oracle.marginalize_window_merge(w.window, v, prm, *args, max_samples=50)
    assert r["status"] == 9  # CGMLI_E_LIMIT
    # a victim whose speed/bias is in the prior keeps the Schur bridge
    wp, prm2, args2 = stream_window(oracle, 64, replace(SPEC, with_prior=True))
    v2 = wp.K - 2
    kinds = [wp.window.prior_block_kind[b] for b in range(wp.window.prior_num_blocks)]
    b = kinds.index(abi.PRIOR_SPEED_BIAS)
    wp.window.prior_block_index[b] = v2
    r = oracle.marginalize_window_merge(wp.window, v2, prm2, *args2)
    assert r["status"] == 0 and r["merge"] == abi.IMU_MERGE_BRIDGE
    # the edges must meet: a gap between them is rejected
    t, rd, rg, t0, t1 = args
    t0b = t0.copy(); t0b[v] += 1
    r = oracle.marginalize_window_merge(w.window, v, prm, t, rd, rg, t0b, t1)
    assert r["status"] == abi.E_INVALID
