"""Builds the in-tree shared libraries.

* ``cgmli-slam_b200/lib/libcgmli_backend.so`` - the sm_100a CUDA kernels and
  the C ABI of ``include/cgmli_backend.h`` (nvcc, ``-gencode
  arch=compute_100a,code=sm_100a``).
* ``cgmli-slam_b200/lib/libcgmli_synth.so`` - the seeded window generator.
* ``oracle/liboracle.so`` - the FP64 CPU oracle (test infrastructure).

Libraries are rebuilt only when a source is newer than the output.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

BACKEND_SOURCES = [PKG / "csrc" / "backend_kernels.cu", PKG / "csrc" / "marginal_kernels.cu", PKG / "csrc" / "backend_host.cu",
                   PKG / "csrc" / "topology.cpp", PKG / "csrc" / "noalloc_eigen.cu", PKG / "csrc" / "imu_preintegration.cu",
                   PKG / "csrc" / "server.cpp"]
BACKEND_HEADERS = [PKG / "csrc" / "device_math.cuh", PKG / "csrc" / "factor_eval.cuh", PKG / "csrc" / "backend_internal.h",
                   PKG / "csrc" / "dense_tiles.cuh", PKG / "csrc" / "imu_preintegration.h",
                   PKG / "csrc" / "topology.h",
                   INCLUDE / "cgmli_backend.h"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-shared",
]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd) + "\n" + proc.stdout + proc.stderr)


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (Path(cand).exists() or cand == "nvcc"):
            return cand
    return "nvcc"


def build_backend(force: bool = False, verbose: bool = False) -> Path:
    out = LIB / "libcgmli_backend.so"
    if force or _stale(out, BACKEND_SOURCES + BACKEND_HEADERS):
        LIB.mkdir(parents=True, exist_ok=True)
        cmd = [nvcc(), *NVCC_FLAGS, f"-I{INCLUDE}", *map(str, BACKEND_SOURCES), "-o", str(out)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd)
    return out


def build_synth(force: bool = False) -> Path:
    out = LIB / "libcgmli_synth.so"
    src = PKG / "synth" / "window_synth.cpp"
    if force or _stale(out, [src, INCLUDE / "cgmli_backend.h"]):
        LIB.mkdir(parents=True, exist_ok=True)
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", f"-I{INCLUDE}", str(src), "-o", str(out)])
    return out


def build_oracle(force: bool = False) -> Path:
    out = ROOT / "oracle" / "liboracle.so"
    src = ROOT / "oracle" / "cgmli_oracle.cpp"
    if force or _stale(out, [src, INCLUDE / "cgmli_backend.h"]):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-pthread", f"-I{INCLUDE}", str(src), "-o", str(out)])
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_oracle(force)
    build_backend(force)


if __name__ == "__main__":
    import sys

    build_all(force="--force" in sys.argv)
    print("built", LIB)
