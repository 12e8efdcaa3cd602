"""Seeded synthetic matrices of the sparse workloads (CSR, sorted columns).

Every generator returns ``(offsets int32[n+1], columns int32[nnz],
values float64[nnz], n_columns)``. Random numbers come from numpy's
counter-based Philox generator, so a (generator, seed) pair names one matrix
on any machine. These are the workload shapes TNL's SpMV / linear-solver
benchmarks are run on here (src/Benchmarks/SpMV/spmv.h, LinearSolvers/);
no public matrix collection is used.
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(seed))


def _from_coo(n, rows, cols, vals, ncols=None):
    """Rows/cols must already be sorted by (row, col)."""
    counts = np.bincount(rows, minlength=n)
    off = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=off[1:])
    if off[-1] > np.iinfo(np.int32).max:
        raise OverflowError("nnz exceeds int32 indices")
    return (off.astype(np.int32), cols.astype(np.int32), vals.astype(np.float64),
            n if ncols is None else ncols)


def _stencil(shape, terms):
    """Assemble a structured-grid operator.

    ``terms`` is a list of (offset tuple, value array over the grid or scalar);
    entries falling outside the grid are dropped (Dirichlet elimination).
    Column order within a row is ascending because the offsets are applied in
    increasing linear-index order.
    """
    dims = len(shape)
    n = int(np.prod(shape))
    strides = [int(np.prod(shape[d + 1:])) for d in range(dims)]  # C order: last index fastest
    idx = np.arange(n, dtype=np.int64)
    coords = np.unravel_index(idx, shape)
    # sort terms by linear offset so columns come out ascending
    terms = sorted(terms, key=lambda t: sum(o * s for o, s in zip(t[0], strides)))
    rows_l, cols_l, vals_l = [], [], []
    for off, val in terms:
        ok = np.ones(n, dtype=bool)
        for d in range(dims):
            c = coords[d] + off[d]
            ok &= (c >= 0) & (c < shape[d])
        lin = sum(o * s for o, s in zip(off, strides))
        r = idx[ok]
        rows_l.append(r)
        cols_l.append(r + lin)
        v = np.broadcast_to(np.asarray(val, dtype=np.float64), (n,))[ok] if np.ndim(val) else np.full(r.size, val)
        vals_l.append(v)
    rows = np.concatenate(rows_l)
    cols = np.concatenate(cols_l)
    vals = np.concatenate(vals_l)
    order = np.lexsort((cols, rows))
    return _from_coo(n, rows[order], cols[order], vals[order])


def poisson2d(nx: int, ny: int | None = None):
    """5-point Laplacian on an nx x ny grid, Dirichlet boundary eliminated:
    4 on the diagonal, -1 to each in-grid neighbour."""
    ny = nx if ny is None else ny
    return _stencil((ny, nx), [((0, 0), 4.0), ((0, -1), -1.0), ((0, 1), -1.0), ((-1, 0), -1.0), ((1, 0), -1.0)])


def laplace3d(n: int):
    """7-point Laplacian on an n^3 grid (6 on the diagonal, -1 off it)."""
    offs = [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 1), (0, 1, 0), (1, 0, 0)]
    return _stencil((n, n, n), [((0, 0, 0), 6.0)] + [(o, -1.0) for o in offs])


def irregular(rows: int, seed: int = 2, mu: float = np.log(12.0), sigma: float = 1.0,
              lo: int = 1, hi: int = 2048, ncols: int | None = None):
    """Rows with log-normal lengths round(exp(N(mu, sigma))) clipped to
    [lo, hi]; columns uniform without repeats inside a row (stored ascending);
    values N(0, 1)."""
    ncols = rows if ncols is None else ncols
    g = rng(seed)
    lengths = np.clip(np.rint(np.exp(g.normal(mu, sigma, rows))), lo, min(hi, ncols)).astype(np.int64)
    nnz = int(lengths.sum())
    row_of = np.repeat(np.arange(rows, dtype=np.int64), lengths)
    cols = g.integers(0, ncols, nnz, dtype=np.int64)
    keys = row_of * ncols + cols
    while True:
        keys.sort()
        dup = np.flatnonzero(keys[1:] == keys[:-1]) + 1
        if dup.size == 0:
            break
        r = keys[dup] // ncols
        keys[dup] = r * ncols + g.integers(0, ncols, dup.size, dtype=np.int64)
    vals = g.normal(0.0, 1.0, nnz)
    return _from_coo(rows, keys // ncols, keys % ncols, vals, ncols)


def diffusion3d(n: int, seed: int = 3):
    """SPD variable-coefficient 7-point diffusion on an n^3 grid: every cell
    face f carries kappa_f = exp(N(0, 1)); A_ii sums the six faces of cell i
    (Dirichlet boundary faces included), A_ij = -kappa of the shared face."""
    g = rng(seed)
    kx = np.exp(g.normal(0.0, 1.0, (n + 1, n, n)))  # faces normal to axis 0
    ky = np.exp(g.normal(0.0, 1.0, (n, n + 1, n)))
    kz = np.exp(g.normal(0.0, 1.0, (n, n, n + 1)))
    diag = kx[:-1] + kx[1:] + ky[:, :-1] + ky[:, 1:] + kz[:, :, :-1] + kz[:, :, 1:]
    terms = [((0, 0, 0), diag.ravel()),
             ((-1, 0, 0), -kx[:-1].ravel()), ((1, 0, 0), -kx[1:].ravel()),
             ((0, -1, 0), -ky[:, :-1].ravel()), ((0, 1, 0), -ky[:, 1:].ravel()),
             ((0, 0, -1), -kz[:, :, :-1].ravel()), ((0, 0, 1), -kz[:, :, 1:].ravel())]
    return _stencil((n, n, n), terms)


def convdiff3d(n: int, peclet: float = 10.0, seed: int = 4):
    """Nonsymmetric 7-point convection-diffusion with first-order upwinding on
    an n^3 grid (unit mesh spacing, unit diffusivity): a random unit velocity
    v scaled so that the cell Peclet number |v| h / D equals ``peclet``.
    Each axis adds peclet*|v_d| to the diagonal and -peclet*|v_d| to the
    upwind neighbour."""
    g = rng(seed)
    v = g.normal(0.0, 1.0, 3)
    v /= np.linalg.norm(v)
    a = peclet * v
    diag = 6.0 + np.abs(a).sum()
    coef = {}
    for d in range(3):
        for s in (-1, 1):
            off = [0, 0, 0]
            off[d] = s
            c = -1.0
            if (a[d] > 0 and s == -1) or (a[d] < 0 and s == 1):
                c -= abs(a[d])
            coef[tuple(off)] = c
    terms = [((0, 0, 0), diag)] + [(o, c) for o, c in coef.items()]
    return _stencil((n, n, n), terms)


def spd_shifted_poisson2d(nx: int, ny: int, shift: float):
    """2D 5-point Laplacian plus a diagonal shift (batched-solve systems)."""
    off, col, val, nc = poisson2d(nx, ny)
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
    val = val.copy()
    val[col == rows] += shift
    return off, col, val, nc


def batched_poisson2d(nsys: int, seed: int = 5, lo: int = 32, hi: int = 256, max_shift: float = 0.1,
                      max_rhs: int = 8):
    """The batched-solve workload: ``nsys`` independent SPD systems, system s a
    5-point Laplacian on an nx_s x ny_s grid (nx, ny uniform in [lo, hi]) plus
    a diagonal shift uniform in [0, max_shift], with 1..max_rhs right-hand
    sides. Returns the block-diagonal CSR (offsets int32[N+1], global column
    indices int32, values) with row_ptr int64[nsys+1] and nrhs int32[nsys].
    Built vectorised over all rows at once."""
    g = rng(seed)
    nx = g.integers(lo, hi + 1, nsys)
    ny = g.integers(lo, hi + 1, nsys)
    shift = g.uniform(0.0, max_shift, nsys)
    nrhs = g.integers(1, max_rhs + 1, nsys).astype(np.int32)
    n_sys = (nx * ny).astype(np.int64)
    row_ptr = np.zeros(nsys + 1, dtype=np.int64)
    np.cumsum(n_sys, out=row_ptr[1:])
    N = int(row_ptr[-1])
    sys_of = np.repeat(np.arange(nsys, dtype=np.int32), n_sys)
    loc = np.arange(N, dtype=np.int64) - row_ptr[sys_of]
    sx = nx[sys_of]
    i = (loc % sx).astype(np.int32)
    j = (loc // sx).astype(np.int32)
    del loc
    has = [j > 0, i > 0, np.ones(N, dtype=bool), i < sx - 1, j < ny[sys_of] - 1]  # ascending column order
    cnt = np.zeros(N, dtype=np.int32)
    for h in has:
        cnt += h
    off = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(cnt, out=off[1:])
    if off[-1] > np.iinfo(np.int32).max:
        raise OverflowError("nnz exceeds int32 indices")
    nnz = int(off[-1])
    col = np.empty(nnz, dtype=np.int32)
    val = np.empty(nnz, dtype=np.float64)
    pos = off[:-1].copy()
    r = np.arange(N, dtype=np.int64)
    deltas = [-sx, -1, 0, 1, sx]
    for h, d in zip(has, deltas):
        idx = np.flatnonzero(h)
        p = pos[idx]
        col[p] = (r[idx] + (d[idx] if isinstance(d, np.ndarray) else d)).astype(np.int32)
        val[p] = (4.0 + shift[sys_of[idx]]) if (not isinstance(d, np.ndarray) and d == 0) else -1.0
        pos[idx] += 1
    return off.astype(np.int32), col, val, row_ptr, nrhs


def uniform(n: int, seed: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    return rng(seed).uniform(lo, hi, n)


def batch_system(off, col, val, row_ptr, s: int):
    """System ``s`` of a block-diagonal batch (``batched_poisson2d``) as a
    stand-alone CSR matrix ``(offsets, columns, values, n)`` with local indices."""
    r0, r1 = int(row_ptr[s]), int(row_ptr[s + 1])
    o0, o1 = int(off[r0]), int(off[r1])
    n = r1 - r0
    return ((np.asarray(off[r0:r1 + 1], dtype=np.int64) - o0).astype(np.int32),
            (np.asarray(col[o0:o1], dtype=np.int64) - r0).astype(np.int32),
            np.asarray(val[o0:o1], dtype=np.float64), n)
