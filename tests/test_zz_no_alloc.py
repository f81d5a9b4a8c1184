"""GPU check of cgmli_marg_eigen_noalloc, the allocation-free eigensolver.

Callers that share the GPU with latency-critical work (cudaFree synchronizes
the device) or whose device memory belongs to another allocator cannot let
the library allocate; this entry point keeps its work arrays in a fixed device
array instead.  The test gives it device buffers (allocated here by the test,
not by the library) and compares its results with cgmli_marg_eigen on the same
matrices, within the dense-eigensolver tolerance of the other tests, on two
calls in a row (the second reuses the shared array left by the first), and
checks that the second call leaves the device's free memory unchanged.
This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cgmli_slam_b200 import abi

pytestmark = pytest.mark.gpu


def _spd(rng, n, rank_deficit=2):
    X = rng.standard_normal((n, max(1, n - rank_deficit)))
    return X @ X.T + np.diag(rng.uniform(0, 1e-3, n))


def _noalloc(lib, torch, H):
    """Runs the entry point on device buffers the test allocates; also returns the device's
    free memory (cudaMemGetInfo) right before and right after the call."""
    n = H.shape[0]
    dH = torch.tensor(np.asfortranarray(H).ravel(order="F"), dtype=torch.float64, device="cuda")
    dev = torch.empty(n, dtype=torch.float64, device="cuda")
    dU = torch.empty(n * n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    code = lib.cgmli_marg_eigen_noalloc(C.c_void_p(dH.data_ptr()), n, C.c_void_p(dev.data_ptr()), C.c_void_p(dU.data_ptr()),
                                        C.c_void_p(stream))
    free1 = torch.cuda.mem_get_info()[0]
    assert code == 0, lib.cgmli_last_error()
    return dev.cpu().numpy(), dU.cpu().numpy().reshape(n, n, order="F"), free0, free1


def test_noalloc_eigen_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    from cgmli_slam_b200 import backend as B

    lib = B.lib()
    rng = np.random.default_rng(11)
    for call, n in enumerate((181, 7)):  # two calls in a row, the second smaller than the first
        H = _spd(rng, n)
        ev_ref, U_ref = B.marg_eigen(H)
        ev, U, free0, free1 = _noalloc(lib, torch, H)
        if call == 1:  # after the set-up call, a call takes no device memory at all
            assert free1 == free0
        scale = np.max(np.abs(ev_ref))
        assert np.max(np.abs(ev - ev_ref)) <= 1e-12 * scale
        # eigenvectors agree up to the sign of each column
        signs = np.sign(np.sum(U * U_ref, axis=0))
        signs[signs == 0] = 1
        assert np.max(np.abs(U * signs - U_ref)) < 1e-12
        assert np.linalg.norm(U @ np.diag(ev) @ U.T - H) / np.linalg.norm(H) < 1e-13


def test_noalloc_eigen_rejects_sizes_above_its_limit():
    torch = pytest.importorskip("torch")
    from cgmli_slam_b200 import backend as B

    lib = B.lib()
    n = abi.MARG_EIGEN_NOALLOC_MAX_N + 1
    buf = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    code = lib.cgmli_marg_eigen_noalloc(C.c_void_p(buf.data_ptr()), n, C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                        None)
    assert code == 9  # CGMLI_E_LIMIT
    assert b"CGMLI_MARG_EIGEN_NOALLOC_MAX_N" in lib.cgmli_last_error()
