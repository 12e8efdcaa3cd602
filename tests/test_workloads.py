"""Seeded workload generators: sizes and structure of the configured matrices."""
import numpy as np

from b2s import workloads as W


def test_poisson2d_256():
    off, col, val, nc = W.poisson2d(256)
    assert len(off) - 1 == 65536 and off[-1] == 326656
    rows = np.repeat(np.arange(65536), np.diff(off))
    assert np.all(val[col == rows] == 4.0) and np.all(val[col != rows] == -1.0)
    # sorted columns in every row
    assert np.all((np.diff(col) > 0) | (np.diff(rows) > 0))


def test_laplace3d_small_matches_formula():
    n = 10
    off, col, val, nc = W.laplace3d(n)
    assert off[-1] == 7 * n**3 - 6 * n**2
    rows = np.repeat(np.arange(n**3), np.diff(off))
    rowsum = np.bincount(rows, weights=val, minlength=n**3)
    # interior rows sum to 0, boundary rows to the number of missing neighbours
    assert rowsum.min() == 0.0 and rowsum.max() == 3.0


def test_irregular_properties():
    off, col, val, nc = W.irregular(20000, seed=2)
    lens = np.diff(off)
    assert lens.min() >= 1 and lens.max() <= 2048
    rows = np.repeat(np.arange(20000), lens)
    # strictly increasing columns inside a row (no repeats)
    assert np.all((np.diff(col) > 0) | (np.diff(rows) > 0))
    assert 15 < lens.mean() < 25
    again = W.irregular(20000, seed=2)
    assert np.array_equal(again[1], col) and np.array_equal(again[2], val)


def test_diffusion3d_is_spd_structure():
    off, col, val, nc = W.diffusion3d(6, seed=3)
    n = 216
    rows = np.repeat(np.arange(n), np.diff(off))
    A = np.zeros((n, n))
    A[rows, col] = val
    assert np.array_equal(A, A.T)
    diag = np.diag(A)
    off_sum = diag - A.sum(axis=1)
    assert np.all(diag >= off_sum - 1e-12)  # weakly diagonally dominant, strictly at the boundary
    assert np.any(diag > off_sum + 1e-12)
    assert np.linalg.eigvalsh(A).min() > 0


def test_convdiff3d_upwind():
    off, col, val, nc = W.convdiff3d(6, peclet=10.0, seed=4)
    rows = np.repeat(np.arange(216), np.diff(off))
    rowsum_interior = np.bincount(rows, weights=val, minlength=216)
    assert np.isclose(rowsum_interior.min(), 0.0, atol=1e-12)  # interior rows conserve
    assert not np.allclose(val[(rows != col)], -1.0)  # nonsymmetric couplings
