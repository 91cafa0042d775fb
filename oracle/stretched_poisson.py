"""Oracle (test infrastructure only) for the cal_w system on a vertically
stretched grid. The reference model has uniform levels only; this file is the
restatement its generalisation is checked against.

The reference's matrix (src/PoissonSolver.cpp:760-796) is, for unknown
W[kk][ii] (kk = k-2, reference ordering kk*NX + ii),

    (A W) = W[i-1] - 2 W[i] + W[i+1] + ru_k (W[k+1] - W[k]) - rd_k (W[k] - W[k-1]),
    ru_k = rhow_k / rhou_k,  rd_k = rhow_k / rhou_{k-1},

dx^2 times the anelastic operator d2/dx2 + rhow d/dz (1/rhou d/dz) when
dx = dz. On levels with face heights z_zeta[k] and centre heights z[k]
(centres midway between faces) the same operator, times dx^2, has

    ru_k = rhow_k h_k / (a_k rhou_k),  rd_k = rhow_k h_{k-1} / (a_k rhou_{k-1}),
    a_k = (z[k] - z[k-1]) / dx    (centre-to-centre distance around face k),
    h_k = dx / (2 (z[k] - z_zeta[k]))   (thickness of centre cell k),

which is the reference's matrix when the levels are uniform and dz = dx.
The right-hand side b = rhow_k^2 (zeta[i+1] - zeta[i]) dx is unchanged
(src/PoissonSolver.cpp:444-450): it has no vertical derivative.
"""
from __future__ import annotations

import numpy as np


def metric(z: np.ndarray, z_zeta: np.ndarray, dx: float) -> tuple[np.ndarray, np.ndarray]:
    """(a, h) on the model's nz levels (1 outside the rows they are used on)."""
    nz = len(z)
    a = np.ones(nz)
    h = np.ones(nz)
    for k in range(2, nz - 1):
        a[k] = (z[k] - z[k - 1]) / dx
    for k in range(1, nz - 1):
        h[k] = dx / (2.0 * (z[k] - z_zeta[k]))
    return a, h


def operator(rhou, rhow, z, z_zeta, dx: float, NX: int):
    """The stretched cal_w matrix as scipy CSR, reference unknown ordering."""
    import scipy.sparse as sp
    nz = len(rhou)
    NK = nz - 3
    a, h = metric(np.asarray(z), np.asarray(z_zeta), dx)
    rows, cols, vals = [], [], []
    for kk in range(NK):
        k = kk + 2
        ru = rhow[k] * h[k] / (a[k] * rhou[k])
        rd = rhow[k] * h[k - 1] / (a[k] * rhou[k - 1])
        for ii in range(NX):
            r = kk * NX + ii
            rows += [r, r, r]
            cols += [r, kk * NX + (ii - 1) % NX, kk * NX + (ii + 1) % NX]
            vals += [-(2.0 + ru + rd), 1.0, 1.0]
            if kk + 1 < NK:
                rows.append(r); cols.append(r + NX); vals.append(ru)
            if kk > 0:
                rows.append(r); cols.append(r - NX); vals.append(rd)
    n = NK * NX
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def rhs(rhow, zetap: np.ndarray, dx: float) -> np.ndarray:
    """b in the reference ordering from a [nx][nz] zeta field."""
    nx, nz = zetap.shape
    out = []
    for k in range(2, nz - 1):
        out.append(rhow[k] * rhow[k] * (zetap[2:nx, k] - zetap[1:nx - 1, k]) * dx)
    return np.concatenate(out)


def solve(A, b: np.ndarray) -> np.ndarray:
    from scipy.sparse.linalg import spsolve
    return spsolve(A.tocsc(), b)
