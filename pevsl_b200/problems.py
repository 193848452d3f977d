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


def laplacian_shifted(nx: int, ny: int, nz: int, shift: float):
    """laplacian(nx, ny, nz) + shift * I: (n, ia, ja, a).  Its eigenvalues
    are those of the Laplacian plus shift."""
    n, ia, ja, a = laplacian(nx, ny, nz)
    a = a.copy()
    rows = np.repeat(np.arange(n), np.diff(ia))
    a[ja == rows] += shift
    return n, ia, ja, a


def _gap_midpoint(ev: np.ndarray, t: float, tol: float = 1e-10) -> float:
    """Midpoint of the gap between distinct eigenvalues (ascending ev) that
    lies nearest to t."""
    j = int(np.clip(np.searchsorted(ev, t), 1, len(ev) - 1))
    best = None
    for jj in range(max(1, j - 64), min(len(ev), j + 64)):
        if ev[jj] - ev[jj - 1] > tol:
            m = 0.5 * (ev[jj - 1] + ev[jj])
            if best is None or abs(m - t) < abs(best - t):
                best = m
    return float(best if best is not None else t)


def multi_laplacian_set(count: int = 32, seed: int = 2024, per_slice: int = 20):
    """The batched-problem workload: `count` Dirichlet Laplacians, each a 2D
    5-point or 3D 7-point grid (coin flip) with equal sides drawn uniformly
    so that n = side^d lies in [1e4, 5e5], plus a diagonal shift drawn from
    U[0, 0.5], and 2..8 slices.  The interval of a problem starts at 0.5%
    of its spectral width above the bottom of the spectrum and holds
    per_slice * nslices eigenvalues; the slices split it about evenly, every
    slice end lying midway between two distinct eigenvalues.  Returns a list of dicts:
    grid, n, shift, nslices, intv (slice ends), lmin, lmax (spectrum bounds
    with a 1e-3 margin), counts (eigenvalues per slice)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        d = 2 if rng.random() < 0.5 else 3
        smin = int(np.ceil(1e4 ** (1.0 / d)))
        smax = int(np.floor(5e5 ** (1.0 / d)))
        s = int(rng.integers(smin, smax + 1))
        shift = float(rng.uniform(0.0, 0.5))
        ns = int(rng.integers(2, 9))
        grid = (s, s, s) if d == 3 else (s, s, 1)
        ev = laplacian_eigenvalues(*grid, 0.0, 100.0)
        lo, hi = ev[0], ev[-1]
        i0 = int(np.searchsorted(ev, lo + 0.005 * (hi - lo)))
        i1 = min(i0 + per_slice * ns, len(ev) - 1)
        # slice ends at gap midpoints between distinct eigenvalues (values
        # closer than 1e-10 count as one), the inner ones nearest the even split
        a = _gap_midpoint(ev, 0.5 * (ev[i0 - 1] + ev[i0]))
        b = _gap_midpoint(ev, 0.5 * (ev[i1 - 1] + ev[i1]))
        edges = np.array([a] + [_gap_midpoint(ev, t) for t in np.linspace(a, b, ns + 1)[1:-1]]
                         + [b])
        counts = [int(np.sum((ev >= edges[k]) & (ev < edges[k + 1]))) for k in range(ns)]
        out.append(dict(grid=grid, n=int(s ** d), shift=shift, nslices=ns,
                        intv=[float(x) + shift for x in edges], lmin=float(lo + shift - 1e-3),
                        lmax=float(hi + shift + 1e-3), counts=counts))
    return out


def random_coef_laplacian(nx: int, ny: int, nz: int, seed: int, lo: float = 0.5, hi: float = 2.0):
    """Dirichlet Laplacian on an nx x ny x nz grid (nz = 1: 2D) whose every
    edge, including the edges to the boundary, has a weight drawn from
    U[lo, hi]: A = sum_e c_e (e_i - e_j)(e_i - e_j)^T over interior edges
    plus c_e e_i e_i^T for boundary edges.  Returns (n, ia, ja, a), rows
    sorted by column."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    diag = np.zeros(n)
    rows, cols, vals = [], [], []
    dims = [(nx, 2), (ny, 1)] + ([(nz, 0)] if nz > 1 else [])
    for size, axis in dims:
        # weights of the size+1 edges along this axis for every grid line
        shape = list(idx.shape)
        shape[axis] = size + 1
        c = rng.uniform(lo, hi, shape)
        lo_sl = [slice(None)] * 3
        hi_sl = [slice(None)] * 3
        lo_sl[axis] = slice(0, size)
        hi_sl[axis] = slice(1, size + 1)
        np.add.at(diag, idx.ravel(), (c[tuple(lo_sl)] + c[tuple(hi_sl)]).ravel())
        # interior edges: between index i and i+1 along the axis, weight c[i+1]
        a_sl = [slice(None)] * 3
        b_sl = [slice(None)] * 3
        w_sl = [slice(None)] * 3
        a_sl[axis] = slice(0, size - 1)
        b_sl[axis] = slice(1, size)
        w_sl[axis] = slice(1, size)
        i = idx[tuple(a_sl)].ravel()
        j = idx[tuple(b_sl)].ravel()
        w = c[tuple(w_sl)].ravel()
        rows += [i, j]
        cols += [j, i]
        vals += [-w, -w]
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    return _coo_to_csr(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def random_sparse_symmetric(n: int, per_row: int, bandwidth: int, seed: int):
    """Symmetric sparse matrix of the general-sparse family: per_row/2
    off-diagonal entries drawn per row at column offsets uniform in
    [1, bandwidth] (either side; draws that fall outside the matrix are
    dropped, so no row collects the overflow), values N(0,1), symmetrised
    as (B + B^T), duplicates summed, plus the diagonal 4 + U[0, 1].  About
    per_row nonzeros per row.  Returns (n, ia, ja, a)."""
    rng = np.random.default_rng(seed)
    h = max(1, per_row // 2)
    i = np.repeat(np.arange(n), h)
    off = rng.integers(1, bandwidth + 1, size=i.size) * np.where(rng.random(i.size) < 0.5, -1, 1)
    j = i + off
    keep = (j >= 0) & (j < n)
    i, j = i[keep], j[keep]
    v = rng.standard_normal(i.size)
    # sum duplicates on the upper triangle, then mirror: exactly symmetric
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    _, iu, ju, vu = _coo_to_csr(n, lo, hi, v)
    ru = np.repeat(np.arange(n), np.diff(iu))
    rows = np.concatenate([ru, ju, np.arange(n)])
    cols = np.concatenate([ju, ru, np.arange(n)])
    vals = np.concatenate([vu, vu, 4.0 + rng.random(n)])
    return _coo_to_csr(n, rows, cols, vals)


def _coo_to_csr(n, rows, cols, vals):
    """CSR (int32 indices, rows sorted by column, duplicates summed)."""
    key = rows.astype(np.int64) * n + cols
    order = np.argsort(key, kind="stable")
    key, vals = key[order], vals[order]
    uniq, start = np.unique(key, return_index=True)
    sums = np.add.reduceat(vals, start)
    r = (uniq // n).astype(np.int64)
    c = (uniq % n).astype(np.int32)
    ia = np.zeros(n + 1, np.int32)
    np.add.at(ia, r + 1, 1)
    ia = np.cumsum(ia).astype(np.int32)
    return n, ia, c, np.ascontiguousarray(sums, dtype=np.float64)
