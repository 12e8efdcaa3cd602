"""Test matrices and closed-form expected products of TNL's own SpMV unit tests,
src/UnitTests/Matrices/SparseMatrixVectorProductTest.hpp, restated as CSR
arrays (every case multiplies by a constant input vector):

* smallMatrix1/2/3            (:17-178)  4x4, x = 2
* mediumSizeMatrix1/2         (:179-338) 8x8, x = 2
* largeMatrix diagonal        (:339-375) 1051x1051, A_ii = i+1, x = 1
* largeMatrix lower triangle  (:376-401) A_ij = j+1 for j <= i, x = 1
* longRowsMatrix              (:403-434) 33 x cols, A_rc = c + r, x = 1
"""
from __future__ import annotations

import numpy as np


def _csr(rows, ncols, entries):
    """entries: list per row of (col, value) in insertion (= ascending) order."""
    off = np.zeros(rows + 1, dtype=np.int32)
    cols, vals = [], []
    for r, row in enumerate(entries):
        row = sorted(row)
        off[r + 1] = off[r] + len(row)
        cols += [c for c, _ in row]
        vals += [v for _, v in row]
    return off, np.array(cols, dtype=np.int32), np.array(vals, dtype=np.float64), ncols


def small1():
    e = [[(0, 1)], [(1, 2), (3, 3)], [(1, 4)], [(2, 5)]]
    return _csr(4, 4, e), 2.0, [2, 10, 8, 10]


def small2():
    e = [[(0, 1), (1, 2), (2, 3)], [(3, 4)], [(0, 5), (1, 6), (2, 7)], [(1, 8)]]
    return _csr(4, 4, e), 2.0, [12, 8, 36, 16]


def small3():
    e = [[(0, 1), (1, 2), (2, 3)], [(1, 4), (2, 5), (3, 6)], [(0, 7), (1, 8), (2, 9)], [(1, 10), (2, 11), (3, 12)]]
    return _csr(4, 4, e), 2.0, [12, 30, 48, 66]


def medium1():
    v = iter(range(1, 100))
    e = [[(0, next(v)), (1, next(v)), (2, next(v)), (5, next(v))],
         [(c, next(v)) for c in range(1, 5)],
         [(c, next(v)) for c in range(0, 5)],
         [(c, next(v)) for c in range(1, 5)],
         [(c, next(v)) for c in range(2, 6)],
         [(c, next(v)) for c in range(3, 7)],
         [(c, next(v)) for c in range(0, 5)],
         [(c, next(v)) for c in range(0, 5)]]
    return _csr(8, 8, e), 2.0, [20, 52, 110, 124, 156, 188, 280, 330]


def medium2():
    v = iter(range(1, 100))
    e = [[(0, next(v)), (1, next(v)), (2, next(v)), (4, next(v)), (5, next(v))],
         [(1, next(v)), (3, next(v))],
         [(1, next(v)), (2, next(v)), (4, next(v))],
         [(c, next(v)) for c in range(1, 5)],
         [(1, next(v))],
         [(c, next(v)) for c in range(1, 7)],
         [(c, next(v)) for c in range(0, 7)],
         [(c, next(v)) for c in range(0, 8)]]
    for r in range(7):
        e[r].append((7, 1))
    return _csr(8, 8, e), 2.0, [32, 28, 56, 102, 32, 224, 352, 520]


def large_diagonal(size=1051):
    e = [[(i, i + 1)] for i in range(size)]
    return _csr(size, size, e), 1.0, [i + 1 for i in range(size)]


def large_triangular(size=1051):
    off = np.zeros(size + 1, dtype=np.int64)
    off[1:] = np.cumsum(np.arange(1, size + 1))
    cols = np.concatenate([np.arange(i + 1) for i in range(size)]).astype(np.int32)
    vals = (cols + 1).astype(np.float64)
    return (off.astype(np.int32), cols, vals, size), 1.0, [(i + 1) * (i + 2) / 2 for i in range(size)]


def long_rows(columns):
    rows = 33
    off = (np.arange(rows + 1, dtype=np.int64) * columns).astype(np.int32)
    cols = np.tile(np.arange(columns, dtype=np.int32), rows)
    vals = (np.tile(np.arange(columns), rows) + np.repeat(np.arange(rows), columns)).astype(np.float64)
    expected = [columns * (columns - 1) / 2.0 + columns * r for r in range(rows)]
    return (off, cols, vals, columns), 1.0, expected


LONG_ROW_COLUMNS = [64, 65, 128, 129, 256, 257, 512, 513, 1024, 1025, 2048, 2049, 3000]


def all_cases():
    cases = {"small1": small1(), "small2": small2(), "small3": small3(), "medium1": medium1(),
             "medium2": medium2(), "large_diagonal": large_diagonal(), "large_triangular": large_triangular()}
    for c in LONG_ROW_COLUMNS:
        cases[f"long_rows_{c}"] = long_rows(c)
    return cases
