#!/usr/bin/env python
"""Window solves/sec of the batched sliding-window backend solve on B200.

Workload (default): the batched configuration - 512 independent windows from
distinct seeds, keyframes U{6..15}, landmarks log-U(200, 5000), track length
2-10, 4-camera rig with per-window extrinsic perturbation (1 cm / 0.3 deg),
IMU factors and a seeded square-root prior, online per-camera extrinsics +
time offset, 5 damped LM iterations per window.  One step = one batched solve
of all windows (device-side LM, no host round trip), started from the same
initial states every step.  Seeded synthetic inputs stand in for the Hilti
2023 replays.

Lines printed (rank 0): one JSON object.  ``--impl reference`` times the
reference algorithm's CPU path instead (the FP64 CPU oracle: the reference's
Ceres/Eigen build cannot be compiled offline).
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent


def _load_package():
    name = "cgmli_slam_b200"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(
            name, ROOT / "cgmli-slam_b200" / "__init__.py", submodule_search_locations=[str(ROOT / "cgmli-slam_b200")])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


_load_package()
import numpy as np  # noqa: E402

from cgmli_slam_b200 import abi, synth  # noqa: E402

METRIC = "window solves/sec"
UNIT = "windows/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--windows", type=int, default=512)
    p.add_argument("--iterations", type=int, default=5)
    p.add_argument("--seed", type=int, default=20260101)
    p.add_argument("--cpu-sample", type=int, default=512,
                   help="windows timed on the host for the CPU baseline and the reference arm (the whole batch by "
                        "default; fewer: every len/n-th window)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--plain-windows", type=int, default=64, help="windows of the batch solved one at a time for the plain path")
    p.add_argument("--marg-steps", type=int, default=3, help="timed batched marginalizations of the solved batch (0: off)")
    p.add_argument("--no-configs", action="store_true", help="skip the single-window configurations c1-c3")
    p.add_argument("--serve-rates", default="5000,10000,20000,50000",
                   help="offered request rates of the served sweep (requests/s, comma separated; empty: off)")
    p.add_argument("--serve-requests", type=int, default=10000, help="requests per served rate (at least 1 s of arrivals)")
    p.add_argument("--serve-pool", type=int, default=512, help="distinct windows the served requests draw from")
    p.add_argument("--calib-steps", type=int, default=2, help="timed calibration-information passes over the solved batch (0: off)")
    p.add_argument("--gate-iterations", type=int, default=10, help="iteration budget of the gated-solve row (0: off)")
    p.add_argument("--imu-rigs", type=int, default=512, help="rigs of the IMU preintegration batch, 11 keyframes each (0: off)")
    p.add_argument("--imu-cpu-sample", type=int, default=1024, help="intervals preintegrated by the oracle for its CPU rate")
    p.add_argument("--mixed-steps", type=int, default=10, help="timed solves of the batch in the other precision (0: off)")
    p.add_argument("--det-steps", type=int, default=5, help="timed solves of the batch with deterministic sums (0: off)")
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                   help="precision of the headline solve, the end-to-end and the served rows (the batched configuration "
                        "states FP32 evaluation with FP64 reduced solves: mixed)")
    return p.parse_args()


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# k_lin_landmark + k_lin_pairs + k_lin_schur DRAM read + write per observation, by
# precision: dram__bytes_read.sum + dram__bytes_write.sum of the three kernels of one
# linearization of the first 64 windows of the batch (451,950 observations) in an ncu
# capture (profiles/lin_traffic_c4x64.md).  Mostly the staged weighted rows (224 bytes
# mixed, 448 FP64) written by the landmark pass and read back in key order.
LIN_DRAM_BYTES_PER_OBS = {"mixed": 910.3, "fp64": 1536.0}
# the landmark pass's limiter (profiles/lin_landmark_mixed_c4x64.md): FP64 pipe and
# issue fractions of the single-kernel capture
LIN_LANDMARK_PROFILE = {"fp64_pipe_pct": 11.6, "issue_active_pct": 22.0, "dram_throughput_pct": 5.1, "warps_active_pct": 13.5,
                        "registers": 168, "top_stall": "long scoreboard (4.4 per issue)"}


def rank_seed(seed: int, rank: int) -> int:
    """Each replica solves its own windows: rank r draws from seed + 100000 r."""
    return seed + 100000 * rank


def max_over_ranks(value: float, dist, device: str = "cuda") -> float:
    """Largest value over all ranks (the job is as slow as its slowest replica)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def min_over_ranks(value: float, dist, device: str = "cuda") -> float:
    """Smallest value over the ranks (a throughput's slowest rank)."""
    return -max_over_ranks(-value, dist, device)


def aggregate_rate(world: int, windows_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job windows/s: every rank's windows over the slowest rank's device time."""
    return world * windows_per_rank * steps / (max_ms / 1000.0)


PRECISION_TEXT = {
    "mixed": "FP64 factor evaluation with its Jacobian blocks and weights rounded to FP32, FP32 staged rows; FP64 residuals, "
             "landmark sums, gradients, reduced system and Cholesky",
    "fp64": "FP64 factor evaluation and accumulation, FP64 Cholesky",
}
DTYPE = {"mixed": "f32+f64", "fp64": "f64"}


def headline_precision(args):
    return abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64


def config_dict(args, world):
    return {
        "workload": "batched windows: K~U{6..15}, L~logU(200,5000), 4 cams, IMU+prior, 24+1 calib, 5 LM it",
        "windows_per_gpu": args.windows, "lm_iterations": args.iterations, "seed": args.seed,
        "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (no flush needed)",
        "precision": PRECISION_TEXT[args.precision],
        "launch": "one CUDA graph per solve, captured on the second solve of the batch and replayed",
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "25"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def window_bytes(w) -> tuple[int, int]:
    """Host bytes uploaded by set_windows for one window, and state bytes read back."""
    W = w.window
    K, E, C, L, F = W.num_keyframes, W.num_extrinsics, W.num_cameras, W.num_landmarks, W.num_observations
    cols = 0
    if W.prior_rank:
        kinds = np.ctypeslib.as_array(W.prior_block_kind, shape=(W.prior_num_blocks,))
        cols = int(sum(9 if k == 1 else 1 if k == 3 else 6 for k in kinds))
        amb = int(sum(9 if k == 1 else 1 if k == 3 else 7 for k in kinds))
    state = 8 * (16 * K + 7 * E + 1 + L)
    h2d = state + 8 * (12 * C) + 4 * C + L * (4 * 4 + 8 * 7) + F * (4 * 2 + 8 * 13) + W.num_imu * (8 * 295 + 4)
    if W.prior_rank:
        h2d += 8 * (W.prior_rank * cols + W.prior_rank + amb) + 8 * W.prior_num_blocks
    return h2d, state


def algorithmic_linearize_bytes(w) -> int:
    """Bytes one linearization must move for a window: observation stream (44 B
    static / 76 B with bearing velocity), landmark stream (28 B), and the
    reduced visual system written once."""
    W = w.window
    moving = W.obs_velocity is not None and bool(W.obs_velocity)
    per_obs = 76 if moving else 44
    K = W.num_keyframes
    ncal = (6 * W.num_extrinsics if W.estimate_extrinsics else 0) + (1 if W.estimate_td else 0)
    npc = 6 * K + ncal
    return per_obs * W.num_observations + 28 * W.num_landmarks + 8 * (npc * (npc + 1) // 2 + 3 * npc)


def peaks():
    try:
        d = json.load(open(ROOT / "MEASURED_PEAKS.json"))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def run_served(args, local, backend):
    """Served mode (the serving configuration), swept over offered rates: requests
    from 128 simulated rigs arrive as a Poisson stream at each rate; each request
    is one LM iteration plus oldest-keyframe marginalization of a window drawn as
    in the batched configuration.  Each trace is replayed by the server's native
    replay (cgmli_server_replay): latency runs from each request's scheduled
    arrival to its completion, so queueing is included; throughput is completed
    requests over the span from the first arrival to the last completion."""
    rates = [float(x) for x in args.serve_rates.split(",") if x.strip()]
    pool = synth.make_windows("c4", args.serve_pool, seed=args.seed + 500)
    rigs = 128
    server = backend.Server(device=local, iterations=1, policy=abi.MARGIN_OLD, precision=headline_precision(args))
    # warm-up: repeated full-pool bursts, so that both solvers reach their working
    # size (growing pinned staging later would synchronize the device mid-trace)
    for _ in range(4):
        server.replay(pool, [0] * len(pool), np.zeros(len(pool)))
    out = []
    for k, rate in enumerate(rates):
        rng = np.random.default_rng(args.seed + 5 + k)
        n_req = max(args.serve_requests, int(rate))
        arrival = np.cumsum(rng.exponential(1.0 / rate, n_req))
        windows = [pool[i % len(pool)] for i in range(n_req)]
        lat, status, span = server.replay(windows, [0] * n_req, arrival)
        lat_sorted = np.sort(lat)
        counts = {}
        for st in status:
            key = abi.ERRORS.get(int(st), int(st))
            counts[key] = counts.get(key, 0) + 1
        out.append({"offered_rate": rate, "throughput": n_req / span, "unit": "requests/s",
                    "p50_ms": float(lat_sorted[n_req // 2]), "p99_ms": float(lat_sorted[min(n_req - 1, int(0.99 * n_req))]),
                    "requests": n_req, "arrival_span_s": float(arrival[-1]), "request_status": counts})
    device_bytes = server.device_bytes()
    server.close()
    return {"rates": out, "rigs": rigs, "memory_budget_bytes": 40 << 30, "device_bytes_held": device_bytes,
            "workload": "1 LM iteration + oldest-keyframe marginalization per request; windows as the batched configuration"}


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _prior_errors(got, ref):
    """A is unique up to an orthogonal transform: compare A^T A and A^T r0."""
    if got.get("status") != 0 or ref.get("status") != 0 or got["rank"] != ref["rank"]:
        return {"status": [got.get("status"), ref.get("status")], "rank": [got.get("rank"), ref.get("rank")]}
    Ag, Ar = got["A"], ref["A"]
    return {"AtA": _rel(Ag.T @ Ag, Ar.T @ Ar), "Atr0": _rel(Ag.T @ got["r0"], Ar.T @ ref["r0"]), "rank": int(got["rank"]),
            "columns": int(got["cols"]), "bar": 1e-8}


def _c2_chain(backend, local, seed):
    """Configuration 2's window: the sixth of a sliding sequence cut from one 15-keyframe
    trajectory, its prior chained from five OLD marginalizations of the windows before it,
    each solved (5 FP64 iterations) and marginalized on the device."""
    long = synth.c2_long_window(seed)
    prior = None
    for i in range(6):
        w = synth.SubWindow(long, i, 10)
        if prior is not None:
            w.set_prior(prior, 1)
        if i == 5:
            return w
        s = backend.Solver(device=local)
        s.set_windows([w])
        s.solve(5)
        s.marginalize([0], abi.MARGIN_OLD)
        s.synchronize()
        s.read_states()
        prior = s.read_prior(0)
        s.close()
        w.store()


def run_configs(args, local, backend):
    """The single-window configurations as stated, each alone on the device:
    c1 (10 KF, 800 landmarks, FP64, 1 LM iteration + OLD marginalization);
    c2 (10 KF, ~3000 landmarks, IMU, 24+1 calibration, prior chained from five
    device marginalizations of the preceding windows; mixed precision, 5
    iterations + OLD); c3 (30 KF, 8 cameras, 20 000 landmarks, mixed precision,
    10 iterations + SECOND_NEW).  Device time of the solve and of the
    marginalization (CUDA events, median of the repetitions); the mixed step dx
    against the FP64 step, the final states against the FP64 oracle, the prior
    against the oracle's; for c3 the linearization's algorithmic GB/s and the
    factorization's FP64 rate from per-kernel CUDA events."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O  # checker of the per-configuration results

    out = {}
    for name, policy, precision in (("c1", abi.MARGIN_OLD, abi.PRECISION_FP64), ("c2", abi.MARGIN_OLD, abi.PRECISION_MIXED),
                                    ("c3", abi.MARGIN_SECOND_NEW, abi.PRECISION_MIXED)):
        it = synth.ITERATIONS[name]
        w = _c2_chain(backend, local, args.seed + 11) if name == "c2" else synth.make_windows(name, 1, seed=args.seed + 11)[0]
        x0 = w.state_vector()
        nr, L = w.retained_dim(), w.L
        row = {"iterations": it, "landmarks": L, "observations": w.window.num_observations, "retained_columns": nr,
               "precision": "mixed" if precision == abi.PRECISION_MIXED else "fp64",
               "marginalization": "OLD" if policy == abi.MARGIN_OLD else "SECOND_NEW"}
        if name == "c2":
            row["prior"] = f"chained from 5 device marginalizations (rank {w.window.prior_rank})"
        victim = 0 if policy == abi.MARGIN_OLD else w.K - 2
        s = backend.Solver(device=local, precision=precision)
        s.set_windows([w])
        s.checkpoint()
        if precision == abi.PRECISION_MIXED:  # first step at lambda 1e-4: mixed against FP64
            s.step(1e-4)
            dm = s.read_step(0)["delta"]
            f64 = backend.Solver(device=local)
            f64.set_windows([w])
            f64.step(1e-4)
            row["step_dx_rel_err_vs_fp64"] = {"all": _rel(dm, f64.read_step(0)["delta"]),
                                              "retained": _rel(dm[:nr], f64.read_step(0)["delta"][:nr]), "bar": 1e-6}
            f64.close()
        solve_ms, marg_ms = [], []
        for rep in range(4):
            s.rollback()
            s.solve(it)
            s.synchronize()
            if rep:
                solve_ms.append(s.timing()[0])
        if name == "c3":  # per-kernel events of one more solve
            s.kernel_times(enable=1)
            s.rollback()
            s.solve(it)
            s.synchronize()
            kt = s.kernel_times(enable=-1)
            s.kernel_times(enable=0)
        rep_dev = s.reports()[0]
        for rep in range(4):
            s.marginalize([victim], policy)
            s.synchronize()
            if rep:
                marg_ms.append(s.timing()[0])
        prior = s.read_prior(0)
        s.read_states()
        xg = w.state_vector()
        s.close()
        ref_prior = O.marginalize_window(w.window, victim, policy)  # at the device's solved states
        w.set_state_vector(x0)
        O.lm_solve(w.window, it)
        xc = w.state_vector()
        w.set_state_vector(x0)
        solve_ms.sort()
        marg_ms.sort()
        row.update({"solve_ms_p50": solve_ms[len(solve_ms) // 2], "solves_per_s": 1000.0 / solve_ms[len(solve_ms) // 2],
                    "marginalization_ms_p50": marg_ms[len(marg_ms) // 2], "accepted_steps": rep_dev.accepted_steps,
                    "final_state_rel_err_vs_fp64_oracle": float(np.linalg.norm(xg - xc) / max(np.linalg.norm(xc - x0), 1e-300)),
                    "prior_rel_err_vs_fp64_oracle": _prior_errors(prior, ref_prior)})
        if name == "c3":
            lin_ms = sum(kt[k][0] for k in ("linearize", "lin_pairs", "lin_schur"))
            lins = kt["linearize"][1]
            fac_ms, fac_launches = kt["factor"]
            facs = kt["candidate"][1]  # one factorization per iteration (k_factor, or the wide sequence's launches)
            flops = nr ** 3 / 3.0 + 2.0 * nr * nr  # Cholesky + the two triangular solves
            row["linearization"] = {"ms_per_launch": lin_ms / max(1, lins),
                                    "algorithmic_GBps": algorithmic_linearize_bytes(w) * lins / (lin_ms / 1e3) / 1e9,
                                    "hbm_peak_GBps": peaks()[0], "launches": lins}
            row["factorization"] = {"ms_per_factorization": fac_ms / max(1, facs), "fp64_GFLOPs": flops * facs / (fac_ms / 1e3) / 1e9,
                                    "fp64_nominal_peak_GFLOPs": 37000.0, "factorizations": facs, "launches": fac_launches,
                                    "flops_per_factorization": flops}
        out[name] = row
    return out


def run_e2e_pipelined(args, local, backend, windows, rank):
    """End to end through the served API (cgmli_server_*): the batch plus three
    more batches of distinct windows drawn the same way (a solved window reused
    would converge faster), all submitted at once, solved with the batch's LM
    iterations and no marginalization.  The server's two solvers overlap each
    batch's host build and upload with the other batch's solve; every request's
    window goes host -> device and its states come back.  Throughput is the
    windows over the span from the first submission to the last completion, so
    the first batch's unoverlapped build is included."""
    extra = synth.make_windows("c4", 3 * args.windows, seed=rank_seed(args.seed, rank) + 7777)
    pool = list(windows) + extra
    init = [w.state_vector() for w in pool]
    server = backend.Server(device=local, iterations=args.iterations, policy=abi.MARGIN_OLD, max_batch_windows=args.windows,
                            precision=headline_precision(args))
    victims = [-1] * len(pool)
    for _ in range(2):  # warm-up: both solvers and their pinned staging reach the batch size
        server.replay(pool, victims, np.zeros(len(pool)))
        for w, x in zip(pool, init):
            w.set_state_vector(x)
    lat, status, span = server.replay(pool, victims, np.zeros(len(pool)))
    for w, x in zip(pool, init):
        w.set_state_vector(x)
    server.close()
    counts = {}
    for st in status:
        k = abi.ERRORS.get(int(st), int(st))
        counts[k] = counts.get(k, 0) + 1
    return len(pool) / span, len(pool), counts


def run_gated(args, local, backend, windows, init):
    """The batch solved with the NIS gate and up to 3 outlier refits
    (cgmli_solver_solve_gated, threshold 9.21, no pre-solve gate: the synthetic
    windows start perturbed), against the plain solve at the same iteration
    budget, both timed on the device.  Rejections persist on the device until
    the next set_windows, so every repetition re-uploads the batch (untimed)."""
    it = args.gate_iterations
    gs = backend.Solver(device=local)
    plain_ms, gated_ms = [], []
    for rep in range(3):
        for w, x in zip(windows, init):
            w.set_state_vector(x)
        gs.set_windows(windows)
        gs.solve(it)
        gs.synchronize()
        if rep:
            plain_ms.append(gs.timing()[0])
        for w, x in zip(windows, init):
            w.set_state_vector(x)
        gs.set_windows(windows)
        gs.solve_gated(it, pre_gate=False)
        gs.synchronize()
        if rep:
            gated_ms.append(gs.timing()[0])
    launches = gs.timing()[1]
    passes, rejected, evaluated = {}, 0, 0
    for i in range(len(windows)):
        g, _ = gs.read_gate(i)
        passes[g.passes] = passes.get(g.passes, 0) + 1
        rejected += g.rejected_total
    statuses = {}
    for r in gs.reports():
        k = abi.ERRORS.get(r.status, r.status)
        statuses[k] = statuses.get(k, 0) + 1
    for w, x in zip(windows, init):
        w.set_state_vector(x)
    gs.close()
    g_ms, p_ms = statistics.median(gated_ms), statistics.median(plain_ms)
    return {"iterations": it, "max_refits": 3, "nis_threshold": 9.210340371976184, "gated_ms": g_ms, "plain_ms": p_ms,
            "gated_windows_per_s": len(windows) / (g_ms / 1e3), "overhead": g_ms / p_ms, "launches": launches,
            "rejected_factors": rejected, "observations": sum(w.window.num_observations for w in windows),
            "windows_by_passes": {str(k): v for k, v in sorted(passes.items())}, "window_status": statuses}


def run_imu(args, local, backend):
    """Batched IMU preintegration: the frozen IMU factor of every keyframe
    interval of args.imu_rigs rigs x 11 keyframes (0.3 s apart, 200 Hz samples,
    so ~62 integration steps per interval), one cgmli_imu_preintegrate call per
    step with host buffers (samples in, frozen factors out).  The reference
    preintegrates on the host, one factor at a time (ImuError::redoPreintegration);
    its CPU rate is the FP64 oracle's on one thread over a sample of the intervals."""
    s = synth.imu_stream(args.imu_rigs, 11, args.seed + 13)
    prm = synth.imu_parameters()
    call = lambda: backend.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges, s.t0_ns, s.t1_ns, s.bias)
    for _ in range(3):
        call()
    kernel_ms, wall_s = [], []
    for _ in range(max(3, args.steps)):
        t0 = time.perf_counter()
        got = call()
        wall_s.append(time.perf_counter() - t0)
        kernel_ms.append(backend.imu_last_timing())
    kernel_ms.sort()
    wall_s.sort()
    k_ms = kernel_ms[len(kernel_ms) // 2]
    e_s = wall_s[len(wall_s) // 2]
    # integration steps: sample pairs from the one holding t0 to the one holding t1
    steps = 0
    for (b, e), t0, t1 in zip(s.ranges, s.t0_ns, s.t1_ns):
        ts = s.time_ns[b:e]
        steps += int(np.searchsorted(ts, t1, side="left")) - int(np.searchsorted(ts, t0, side="right")) + 1
    lo, hi = int(s.ranges[:, 0].min()), int(s.ranges[:, 1].max())
    h2d = (hi - lo) * (8 + 48) + s.count * (8 + 8 + 8 + 48)
    d2h = s.count * (C.sizeof(abi.FrozenImu) + 4)
    out = {"intervals": s.count, "steps": steps, "kernel_ms_p50": k_ms, "intervals_per_s": s.count / (k_ms / 1e3),
           "ns_per_step": k_ms * 1e6 / steps,
           "e2e": {"value": s.count / e_s, "unit": "intervals/s", "ms_p50": e_s * 1e3, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h},
           "fp64_gflops_covariance": 4320.0 * steps / (k_ms / 1e3) / 1e9,
           "workload": f"{args.imu_rigs} rigs x 11 keyframes, 0.3 s intervals at 200 Hz"}
    if args.imu_cpu_sample > 0:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O  # cpu_baseline leg and checker of the device factors

        n = min(args.imu_cpu_sample, s.count)
        t0 = time.perf_counter()
        st, ref = O.imu_preintegrate(prm, s.time_ns, s.readings, s.ranges[:n], s.t0_ns[:n], s.t1_ns[:n], s.bias[:n])
        cpu_s = time.perf_counter() - t0
        worst = {"deltas_jacobians": 0.0, "information": 0.0}
        for i in range(n):
            for name in ("delta_quaternion", "delta_velocity", "delta_position", "rotation_gyro", "velocity_gyro",
                         "position_gyro", "velocity_accel", "position_accel"):
                a, b = np.array(getattr(got[i], name)), np.array(getattr(ref[i], name))
                worst["deltas_jacobians"] = max(worst["deltas_jacobians"], float(np.linalg.norm(a - b) / np.linalg.norm(b)))
            Wg = np.array(got[i].whitening).reshape(15, 15, order="F")
            Wr = np.array(ref[i].whitening).reshape(15, 15, order="F")
            Ig, Ir = Wg.T @ Wg, Wr.T @ Wr
            worst["information"] = max(worst["information"], float(np.linalg.norm(Ig - Ir) / np.linalg.norm(Ir)))
        out["cpu_baseline"] = {"value": n / cpu_s, "unit": "intervals/s", "cores": 1, "kind": "port",
                               "sample": f"first {n} intervals, FP64 oracle (four dP/dsigma propagations, dense 15x15)"}
        out["rel_err_vs_fp64_oracle_max"] = worst
    return out


def run_deterministic(args, local, backend, windows, init, solver, dist):
    """The batch with deterministic sums (cgmli_tuning.deterministic = 1): device time of
    the same solve at the headline precision, its pair and Schur pass times, and what
    it buys: two solves give the same bits, and the batch's first window solved alone
    gives the same bits as inside the batch."""
    prec = abi.PRECISION_MIXED if args.precision == "mixed" else abi.PRECISION_FP64
    for w, x in zip(windows, init):
        w.set_state_vector(x)
    det = backend.Solver(device=local, precision=prec)
    tuning = {k: v for k, v in solver.get_tuning().items() if k != "ms"}
    det.set_tuning(**dict(tuning, deterministic=1))
    det.set_windows(windows)
    det.checkpoint()
    for _ in range(max(3, args.warmup)):
        det.rollback()
        det.solve(args.iterations)
        det.synchronize()
    ms = []
    for _ in range(args.det_steps):
        det.rollback()
        det.solve(args.iterations)
        det.synchronize()
        ms.append(det.timing()[0])
    det.kernel_times(enable=1)
    for _ in range(args.det_steps):
        det.rollback()
        det.solve(args.iterations)
        det.synchronize()
    kt = det.kernel_times(enable=-1)
    det.kernel_times(enable=0)
    total = max_over_ranks(sum(ms), dist)
    runs = []
    for _ in range(2):
        det.rollback()
        det.solve(args.iterations)
        det.synchronize()
        det.read_states()
        runs.append([w.state_vector().copy() for w in windows])
    repeat_bitwise = all(np.array_equal(a, b) for a, b in zip(*runs))
    # the atomic form twice: its run-to-run drift is the scale of the difference
    # between the two forms (the same arithmetic in another order of additions)
    atomic = []
    for _ in range(2):
        solver.rollback()
        solver.solve(args.iterations)
        solver.synchronize()
        solver.read_states()
        atomic.append([w.state_vector().copy() for w in windows])

    def worst(xs, ys):
        return max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)) for a, b in zip(xs, ys))
    det.close()
    windows[0].set_state_vector(init[0])
    alone = backend.Solver(device=local, precision=prec)
    alone.set_tuning(**dict(tuning, deterministic=1))
    alone.set_windows([windows[0]])
    alone.solve(args.iterations)
    alone.synchronize()
    alone.read_states()
    alone_bitwise = bool(np.array_equal(windows[0].state_vector(), runs[0][0]))
    alone.close()
    for w, x in zip(windows, init):
        w.set_state_vector(x)
    solver.rollback()
    # lin_schur holds the Schur pass and the slot reduction (k_det_reduce)
    per = {n: kt[n][0] / args.det_steps for n in ("lin_pairs", "lin_schur")}
    return {"windows_per_s": args.windows * len(ms) / (total / 1e3), "ms_per_step": total / len(ms), "steps": len(ms),
            "kernel_ms_per_step": per, "repeat_bitwise": repeat_bitwise, "alone_equals_batch_bitwise": alone_bitwise,
            "state_rel_vs_atomic_max": worst(runs[0], atomic[0]), "atomic_repeat_state_rel_max": worst(atomic[1], atomic[0])}


def run_mixed(args, local, backend, windows, init, solver, dist):
    """The batch in the other precision (FP64 when the headline is mixed): device time
    of the same solve, and the mixed form's accuracy against FP64 (first step dx of
    every window, final states after the solve)."""
    for w, x in zip(windows, init):
        w.set_state_vector(x)
    other_prec = abi.PRECISION_FP64 if args.precision == "mixed" else abi.PRECISION_MIXED
    other = backend.Solver(device=local, precision=other_prec)
    other.set_tuning(**{k: v for k, v in solver.get_tuning().items() if k != "ms"})
    other.set_windows(windows)
    other.checkpoint()
    mixed, f64 = (solver, other) if args.precision == "mixed" else (other, solver)
    # first LM step at lambda = 1e-4 from the initial states, both precisions
    solver.rollback()
    solver.step(1e-4)
    other.step(1e-4)
    dx_retained, dx_all = 0.0, 0.0
    for i, w in enumerate(windows):
        nr = w.retained_dim()
        a, b = mixed.read_step(i)["delta"], f64.read_step(i)["delta"]
        dx_retained = max(dx_retained, float(np.linalg.norm(a[:nr] - b[:nr]) / max(np.linalg.norm(b[:nr]), 1e-300)))
        dx_all = max(dx_all, float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))
    for _ in range(max(3, args.warmup)):
        other.rollback()
        other.solve(args.iterations)
        other.synchronize()
    ms = []
    for _ in range(args.mixed_steps):
        other.rollback()
        other.solve(args.iterations)
        other.synchronize()
        ms.append(other.timing()[0])
    other.kernel_times(enable=1)
    for _ in range(args.mixed_steps):
        other.rollback()
        other.solve(args.iterations)
        other.synchronize()
    kt = other.kernel_times(enable=-1)
    other.kernel_times(enable=0)
    total = max_over_ranks(sum(ms), dist)
    # final states of both precisions, relative to the states
    f64.rollback()
    f64.solve(args.iterations)
    f64.synchronize()
    f64.read_states()
    x64 = [w.state_vector() for w in windows]
    c64 = [r.final_cost for r in f64.reports()]
    a64 = [r.accepted_steps for r in f64.reports()]
    mixed.rollback()
    mixed.solve(args.iterations)
    mixed.synchronize()
    mixed.read_states()
    same = [i for i, r in enumerate(mixed.reports()) if r.accepted_steps == a64[i]]
    state_err = max(float(np.linalg.norm(windows[i].state_vector() - x64[i]) / np.linalg.norm(x64[i])) for i in same)
    cost_err = max(abs(mixed.reports()[i].final_cost - c64[i]) / abs(c64[i]) for i in same)
    statuses = {}
    for r in other.reports():
        key = abi.ERRORS.get(r.status, r.status)
        statuses[key] = statuses.get(key, 0) + 1
    for w, x in zip(windows, init):
        w.set_state_vector(x)
    solver.rollback()
    other.close()
    other_name = "fp64" if args.precision == "mixed" else "mixed"
    return {"precision": other_name, "windows_per_s": args.windows * len(ms) / (total / 1e3), "ms_per_step": total / len(ms),
            "steps": len(ms),
            "mixed_step_dx_rel_err_vs_fp64_max": {"retained": dx_retained, "all": dx_all, "bar": 1e-6},
            "mixed_final_vs_fp64_max": {"state_rel": state_err, "cost_rel": cost_err, "windows_compared": len(same),
                                        "windows_with_other_accept_count": len(windows) - len(same)},
            "window_status": statuses,
            "kernel_ms_per_step": {k: v[0] / len(ms) for k, v in kt.items()},
            "precision_detail": PRECISION_TEXT[other_name]}


def strided_sample(windows, n):
    """Every (len / n)-th window of the batch, from the offset whose sample has the mean
    observation count closest to the batch's, so that the CPU sample has the batch's size
    distribution; returns the indices and a size summary of sample and batch."""
    stride = max(1, len(windows) // max(1, n))
    F = np.array([w.window.num_observations for w in windows], dtype=np.float64)
    # the offset whose sample's mean observation count is closest to the batch's
    offset = min(range(stride), key=lambda o: abs(F[o::stride][:n].mean() - F.mean()))
    idx = list(range(offset, len(windows), stride))[:n]

    def summary(ws):
        L = np.array([w.window.num_landmarks for w in ws])
        K = np.array([w.window.num_keyframes for w in ws])
        F = np.array([w.window.num_observations for w in ws])
        return {"windows": len(ws), "landmarks_p10_p50_p90": [int(np.percentile(L, q)) for q in (10, 50, 90)],
                "keyframes_mean": round(float(K.mean()), 2), "observations_mean": round(float(F.mean()), 1)}

    return idx, {"stride": stride, "offset": offset, "sample": summary([windows[i] for i in idx]), "batch": summary(windows)}


def sample_words(info, total):
    n = info["sample"]["windows"]
    return f"all {n} windows" if n == total else f"{n} windows (every {info['stride']}th of {total})"


def run_reference(args, world, rank):
    """CPU path of the reference algorithm on the host cores (FP64 oracle)."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O  # CPU arm: the only place bench.py runs the oracle besides cpu_baseline

    threads = os.cpu_count() or 1
    batch = synth.make_windows("c4", args.windows, seed=args.seed)
    idx, dist_info = strided_sample(batch, max(1, min(args.cpu_sample, args.windows)))
    # largest window first: the oracle's threads take windows in array order, so this
    # keeps the last ones from running alone (the best schedule for the CPU arm)
    idx = sorted(idx, key=lambda i: -batch[i].window.num_observations)
    windows = [batch[i] for i in idx]
    n = len(windows)
    init = [w.state_vector() for w in windows]
    arr = synth.window_array(windows)
    for _ in range(max(0, min(args.warmup, 1))):
        O.lm_solve_batch(arr, n, args.iterations, threads)
        for w, x in zip(windows, init):
            w.set_state_vector(x)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        st, reps = O.lm_solve_batch(arr, n, args.iterations, threads)
        times.append(time.perf_counter() - t0)
        for w, x in zip(windows, init):
            w.set_state_vector(x)
    total = sum(times)
    value = n * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_dict(args, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sample_words(dist_info, args.windows)} of the batched workload per step, largest first, "
                                   f"{args.iterations} LM iterations, FP64 oracle",
                         "sample_sizes": dist_info},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference Ceres/Eigen CPU path cannot be built offline; the FP64 C++ restatement runs on all host threads",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    from cgmli_slam_b200 import backend

    windows = synth.make_windows("c4", args.windows, seed=rank_seed(args.seed, rank))
    init = [w.state_vector() for w in windows]
    solver = backend.Solver(device=local, precision=headline_precision(args))
    # the work decomposition comes from the autotuner (timed on this batch); it
    # leaves the batch set with the fastest one
    tuning = solver.autotune(windows, args.iterations)
    solver.checkpoint()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # warm-up
    for _ in range(max(3, args.warmup)):
        solver.rollback()
        solver.solve(args.iterations)
        solver.synchronize()
    # timed region: device time per step from CUDA events on the solver's stream;
    # the solve replays the CUDA graph captured on the second warm-up solve
    barrier()
    dev_ms = []
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solver.rollback()
            solver.solve(args.iterations)
            solver.synchronize()
            dev_ms.append(solver.timing()[0])
        barrier()
        wall = time.perf_counter() - t0
    launches = solver.timing()[1] * args.steps
    # per-kernel breakdown: the same solves once more with an event around every
    # kernel (eager launches: per-kernel events do not apply to a graph replay)
    solver.kernel_times(enable=1)
    for _ in range(args.steps):
        solver.rollback()
        solver.solve(args.iterations)
        solver.synchronize()
    ktimes = solver.kernel_times(enable=-1)
    solver.kernel_times(enable=0)
    reports = solver.reports()
    total_ms = max_over_ranks(sum(dev_ms), dist)
    value = aggregate_rate(world, args.windows, args.steps, total_ms)

    # roofline of the linearization (landmark pass + J^T J pass + Schur term): the
    # dominant stage; its algorithmic bytes are the observation and landmark streams
    # read once and the reduced visual system written once
    lin_kernels = ("linearize", "lin_pairs", "lin_schur")
    lin_ms = sum(ktimes[k][0] for k in lin_kernels)
    lin_calls = ktimes["linearize"][1]
    lin_passes = sum(r.iterations for r in reports)  # window-linearizations per solve
    bytes_per_solve = sum(algorithmic_linearize_bytes(w) * r.iterations for w, r in zip(windows, reports))
    achieved = bytes_per_solve * args.steps / (lin_ms / 1000.0) / 1e9 if lin_ms > 0 else 0.0
    peak, peak_kind = peaks()
    # DRAM traffic of one linearization launch over the batch: the per-observation
    # read + write bytes of the three kernels in an ncu capture of the first 64
    # windows (451,950 observations), scaled by this batch's observations
    traffic = LIN_DRAM_BYTES_PER_OBS[args.precision] * sum(w.window.num_observations for w in windows)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": "ncu dram bytes of the three kernels on the first 64 windows, per observation, "
                                                      "scaled by this batch's observations",
                "limiter": "FP64 issue and dependent-load latency, not HBM: the landmark pass's single-kernel capture",
                "landmark_pass_profile": LIN_LANDMARK_PROFILE,
                "algorithmic_bytes_per_launch": bytes_per_solve / max(1, args.iterations),
                "kernel": "k_lin_landmark + k_lin_pairs + k_lin_schur", "peak_source": peak_kind,
                "launch_avg_ms": lin_ms / max(1, lin_calls), "window_linearizations_per_step": lin_passes,
                "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()}}

    # batched marginalization of the solved windows: oldest keyframe, OLD policy,
    # device time of the whole formation (CUDA events on the solver's stream)
    marg = None
    if args.marg_steps > 0:
        mms = []
        for it in range(1 + args.marg_steps):
            solver.marginalize([0] * args.windows, abi.MARGIN_OLD)
            solver.synchronize()
            if it > 0:
                mms.append(solver.timing()[0])
        marg_ms = max_over_ranks(sum(mms) / len(mms), dist)
        marg = {"ms": marg_ms, "windows_per_s": world * args.windows / (marg_ms / 1e3), "launches": solver.timing()[1],
                "workload": "Schur-complement prior of every window of the solved batch, oldest keyframe (OLD)"}

    # conditional calibration information of every solved window (prior included),
    # device time of the whole batched call
    calib = None
    if args.calib_steps > 0:
        cms = []
        for it in range(1 + args.calib_steps):
            solver.calibration_information(include_prior=True)
            solver.synchronize()
            if it > 0:
                cms.append(solver.timing()[0])
        ok = sum(1 for i in range(args.windows) if solver.read_calibration_information(i)["status"] == 0)
        calib_ms = max_over_ranks(sum(cms) / len(cms), dist)
        calib = {"ms": calib_ms, "windows_per_s": world * args.windows / (calib_ms / 1e3), "windows_ok": ok,
                 "launches": solver.timing()[1],
                 "workload": "conditional information of the calibration blocks of every solved window, prior included"}

    # end to end through the C ABI with host buffers: topology + upload, solve, read back
    h2d = sum(window_bytes(w)[0] for w in windows)
    d2h = sum(window_bytes(w)[1] for w in windows)
    e2e_times = []
    e2e_solver = backend.Solver(device=local, precision=headline_precision(args))
    e2e_solver.set_tuning(**{k: v for k, v in tuning.items() if k != "ms"})
    for it in range(1 + max(1, args.steps // 2)):
        for w, x in zip(windows, init):
            w.set_state_vector(x)
        barrier()
        t1 = time.perf_counter()
        e2e_solver.set_windows(windows)
        e2e_solver.solve(args.iterations)
        e2e_solver.synchronize()
        e2e_solver.read_states()
        dt = time.perf_counter() - t1
        if it > 0:
            e2e_times.append(dt)
    e2e_s = max_over_ranks(sum(e2e_times) / len(e2e_times), dist)
    sequential = {"value": world * args.windows / e2e_s, "unit": UNIT,
                  "includes": "one solver: host topology build + H2D of all window data + device LM + D2H of states, in sequence"}
    pipe_rate, pipe_windows, pipe_status = run_e2e_pipelined(args, local, backend, windows, rank)
    pipe_rate = world * min_over_ranks(pipe_rate, dist)
    e2e = {"value": pipe_rate, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "includes": f"served API, {pipe_windows} distinct windows submitted at once in batches of {args.windows}: host build + "
                       "H2D of each window's data + device LM + D2H of its states; two solvers overlap one batch's host work "
                       "with the other's solve",
           "request_status": pipe_status, "sequential": sequential}

    # plain single-window path on equal work: windows of this batch (drawn as the
    # batched configuration), solved one at a time with the same iterations
    plain = None
    if rank == 0 and args.plain_windows > 0:
        pw = windows[:args.plain_windows]
        ps = backend.Solver(device=local, precision=headline_precision(args))
        lat = []
        for i, w in enumerate(pw):
            w.set_state_vector(init[i])
            ps.set_windows([w])
            ps.checkpoint()
            for rep in range(2):
                ps.rollback()
                ps.solve(args.iterations)
                ps.synchronize()
                if rep == 1:
                    lat.append(ps.timing()[0])
            w.set_state_vector(init[i])
        ps.close()
        lat.sort()
        plain = {"windows_per_s": 1000.0 / statistics.mean(lat), "p50_ms": lat[len(lat) // 2],
                 "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))], "windows": len(lat),
                 "workload": f"the first {len(lat)} windows of the batch, each solved alone ({args.iterations} LM iterations, "
                             f"{args.precision}, as the batched value)"}

    served = run_served(args, local, backend) if rank == 0 and args.serve_rates.strip() else None
    configs = run_configs(args, local, backend) if rank == 0 and not args.no_configs else None
    imu = run_imu(args, local, backend) if rank == 0 and args.imu_rigs > 0 else None
    gated = run_gated(args, local, backend, windows, init) if rank == 0 and args.gate_iterations > 0 else None
    mixed = run_mixed(args, local, backend, windows, init, solver, dist) if args.mixed_steps > 0 else None
    deterministic = run_deterministic(args, local, backend, windows, init, solver, dist) if args.det_steps > 0 else None

    statuses = {}
    for r in reports:
        statuses[abi.ERRORS.get(r.status, r.status)] = statuses.get(abi.ERRORS.get(r.status, r.status), 0) + 1

    cpu_baseline = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O  # cpu_baseline leg

        threads = os.cpu_count() or 1
        idx, dist_info = strided_sample(windows, max(1, min(args.cpu_sample, args.windows)))
        idx = sorted(idx, key=lambda i: -windows[i].window.num_observations)  # largest first (see run_reference)
        n = len(idx)
        sample = [windows[i] for i in idx]
        for i in idx:
            windows[i].set_state_vector(init[i])
        arr = synth.window_array(sample)
        t2 = time.perf_counter()
        st, reps = O.lm_solve_batch(arr, n, args.iterations, threads)
        cpu_s = time.perf_counter() - t2
        # states of the same windows solved on the GPU, against the FP64 oracle
        gpu_states = []
        solver.rollback()
        solver.solve(args.iterations)
        solver.synchronize()
        cpu_states = [w.state_vector() for w in sample]
        solver.read_states()
        errs = []
        for w, xc, x0 in zip(sample, cpu_states, [init[i] for i in idx]):
            xg = w.state_vector()
            errs.append(float(np.linalg.norm(xg - xc) / max(np.linalg.norm(xc - x0), 1e-300)))
        for w, x in zip(windows, init):
            w.set_state_vector(x)
        cpu_baseline = {"value": n / cpu_s, "unit": UNIT, "cores": threads, "kind": "port",
                        "sample": f"{sample_words(dist_info, args.windows)} of the batch, largest first, "
                                  f"{args.iterations} LM iterations, FP64 oracle on {threads} threads",
                        "sample_sizes": dist_info, "final_state_rel_err_vs_fp64_max": max(errs)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": DTYPE[args.precision], "data": "synthetic", "config": dict(config_dict(args, world), tuning=tuning),
            "clocks": clocks.summary(), "e2e": e2e, "gpu_launches": launches, "roofline": roofline,
            "cpu_baseline": cpu_baseline, "plain_path": plain,
            "served_vs_plain": (value / world) / plain["windows_per_s"] if plain else None,
            "served": served, "marginalization": marg, "configs": configs, "imu_preintegration": imu,
            "nis_gate": gated, "calibration_information": calib, "other_precision": mixed, "deterministic": deterministic,
            "batch_latency_ms": {"p50": sorted(dev_ms)[len(dev_ms) // 2], "p99": max(dev_ms)},
            "window_status": statuses, "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    e2e_solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
