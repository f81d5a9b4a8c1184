"""Generates the golden fixtures under tests/golden/ with numpy float64.

normal_384x8.npz restates the deterministic fixture of the reference's
parallelNormalEquationsPreservePrior (src/backend/tests/ManagedWindowRegression.cpp:279-309):
J(384x8) = sin(0.011 (row+1)(col+1)), r = linspace(-0.15, 0.4, 384), Huber 1 on the
whole 384-dimensional residual (Ceres corrector: both rows scaled by sqrt(rho')).
Expected robust normal equations and the Schur prior after eliminating
columns 0..3, computed independently of the oracle.

Run: python tests/golden/make_golden.py
"""
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def normal_384x8():
    rows, cols = np.meshgrid(np.arange(384), np.arange(8), indexing="ij")
    J = np.sin(0.011 * (rows + 1) * (cols + 1))
    r = np.linspace(-0.15, 0.4, 384)
    s = float(r @ r)
    delta = 1.0
    rho1 = delta / np.sqrt(s) if s > delta * delta else 1.0  # Huber rho'
    H = rho1 * J.T @ J
    g = rho1 * J.T @ r
    robust = delta * (np.sqrt(s) - 0.5 * delta) if s > delta * delta else 0.5 * s
    m, k = np.arange(4), np.arange(4, 8)
    Hmm, Hmr, Hrr = H[np.ix_(m, m)], H[np.ix_(m, k)], H[np.ix_(k, k)]
    w, U = np.linalg.eigh(0.5 * (Hmm + Hmm.T))
    cut = max(1e-12, 1e-9 * max(0.0, w.max()))
    inv = np.where(w > cut, 1.0 / np.where(w > cut, w, 1.0), 0.0)
    X = U @ np.diag(inv) @ U.T @ np.hstack([Hmr, g[m, None]])
    Hp = Hrr - Hmr.T @ X[:, :4]
    Hp = 0.5 * (Hp + Hp.T)
    bp = g[k] - Hmr.T @ X[:, 4]
    np.savez(HERE / "normal_384x8.npz", J=J, r=r, H=H, g=g, robust_cost=robust, H_prior=Hp, b_prior=bp)


if __name__ == "__main__":
    normal_384x8()
    print("wrote", HERE / "normal_384x8.npz")
