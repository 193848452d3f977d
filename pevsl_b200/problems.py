"""Synthetic problems of the slicing workloads (the role of the reference's
TESTS/COMMON: LocalLapGen, ExactEigLap3).  Host numpy, CSR with int32
indices; the matrix is handed to pevsl_b200.Matrix.from_csr (or to
pEVSL_ParcsrSetup from C).
"""
from __future__ import annotations

import numpy as np


def laplacian(nx: int, ny: int, nz: int):
    """Dirichlet Laplacian on an nx x ny x nz grid: 7-point stencil (diagonal
    6, neighbours -1), or 5-point (diagonal 4) when nz == 1.  Rows in natural
    order, columns ascending within a row (TESTS/COMMON/lapl.c:4-70).
    Returns (n, ia, ja, a)."""
    n = nx * ny * nz
    idx = np.arange(n, dtype=np.int64)
    k = idx // (nx * ny)
    i = (idx - k * nx * ny) // nx
    j = idx - k * nx * ny - i * nx
    diag = 6.0 if nz > 1 else 4.0
    stencil = [(-nx * ny, k > 0), (-nx, i > 0), (-1, j > 0), (0, None), (1, j < nx - 1),
               (nx, i < ny - 1), (nx * ny, k < nz - 1)]
    if nz == 1:
        stencil = [s for s in stencil if abs(s[0]) != nx * ny or s[0] == 0]
    cols = np.stack([idx + o for o, _ in stencil], axis=1)
    mask = np.stack([np.ones(n, bool) if m is None else m for _, m in stencil], axis=1)
    vals = np.where(np.array([o for o, _ in stencil]) == 0, diag, -1.0)
    counts = mask.sum(axis=1)
    ia = np.zeros(n + 1, dtype=np.int32)
    ia[1:] = np.cumsum(counts)
    ja = cols[mask].astype(np.int32)
    a = np.broadcast_to(vals, cols.shape)[mask].astype(np.float64)
    return n, ia, ja, np.ascontiguousarray(a)


def laplacian_eigenvalues(nx: int, ny: int, nz: int, a: float, b: float) -> np.ndarray:
    """All eigenvalues of laplacian(nx, ny, nz) in [a - eps, b + eps],
    ascending: 4 (sin^2(i pi/2(nx+1)) + ...) (TESTS/COMMON/lapl.c:139-169)."""
    eps = np.finfo(np.float64).eps
    tx = np.sin(np.arange(1, nx + 1) * 0.5 * np.pi / (nx + 1.0))
    ty = np.sin(np.arange(1, ny + 1) * 0.5 * np.pi / (ny + 1.0))
    tz = np.sin(np.arange(1, nz + 1) * 0.5 * np.pi / (nz + 1.0)) if nz > 1 else np.zeros(1)
    ev = (4 * (tx[:, None, None] ** 2 + ty[None, :, None] ** 2 + tz[None, None, :] ** 2)).ravel()
    return np.sort(ev[(ev >= a - eps) & (ev <= b + eps)])
