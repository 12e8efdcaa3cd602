"""Batched Jacobi-PCG in one persistent launch (include/b2s.h "Batched solves").

* every system and right-hand side matches the single-system CG solver of this
  library (TNL's CG recurrence with the Diagonal preconditioner) at
  convergence residue 1e-12: solutions within 1e-8 relative, iteration counts
  within 2;
* a system with k right-hand sides gives, bit for bit, what the same
  system gives for each right-hand side alone (each one's arithmetic and
  reduction order do not depend on k);
* every cluster size (1, 2, 4, 8 SMs per system) agrees to 1e-9 relative;
* the autotuner picks one of them and the batch converges to 1e-8.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(nsys=24, seed=3, lo=8, hi=48):
    from b2s import workloads as W
    return W.batched_poisson2d(nsys, seed=seed, lo=lo, hi=hi)


def _vectors(cuda, bt, seed=0):
    g = np.random.default_rng(seed)
    B = g.uniform(-1, 1, bt.vector_length)
    return cuda.tensor(B, device="cuda"), cuda.zeros(bt.vector_length, dtype=cuda.float64, device="cuda")


def test_batch_matches_single_system_solver(b2s_lib, cuda):
    off, col, val, rp, nr = _batch()
    bt = b2s_lib.BatchedCG(off, col, val, rp, nr, tol=1e-12, cluster_size=1)
    B, X = _vectors(cuda, bt)
    assert bt.solve(B, X)
    its, res, sts = bt.results()
    Bh, Xh = B.cpu().numpy(), X.cpu().numpy()
    for s in range(len(nr)):
        r0, r1 = int(rp[s]), int(rp[s + 1])
        n, k = r1 - r0, int(nr[s])
        o0, o1 = int(off[r0]), int(off[r1])
        csr = ((off[r0:r1 + 1] - o0).astype(np.int32), (col[o0:o1] - r0).astype(np.int32), val[o0:o1], n)
        A = b2s_lib.SparseMatrix.from_csr(*csr[:3], n)
        cgs = b2s_lib.CG()
        cgs.setMatrix(A)
        cgs.setPreconditioner("diagonal")
        cgs.setConvergenceResidue(1e-12)
        blk = slice(int(bt.vec_off[s]), int(bt.vec_off[s + 1]))
        for j in range(k):
            b = np.ascontiguousarray(Bh[blk].reshape(n, k)[:, j])
            x = np.zeros(n)
            assert cgs.solve(b, x)
            xb = Xh[blk].reshape(n, k)[:, j]
            err = np.max(np.abs(xb - x)) / np.max(np.abs(x))
            assert err <= 1e-8, (s, j, err)
            slot = int(bt.rhs_off[s]) + j
            assert abs(int(its[slot]) - cgs.getIterations()) <= 2, (s, j, its[slot], cgs.getIterations())
            assert sts[slot] == b2s_lib.OK


def test_rhs_are_independent_bitwise(b2s_lib, cuda):
    off, col, val, rp, nr = _batch(nsys=6, seed=4)
    multi = b2s_lib.BatchedCG(off, col, val, rp, nr, tol=1e-10, cluster_size=2)
    B, X = _vectors(cuda, multi, seed=1)
    multi.solve(B, X)
    ones = np.ones(len(nr), np.int32)
    Bh, Xh = B.cpu().numpy(), X.cpu().numpy()
    for j in range(int(nr.max())):
        sel = [s for s in range(len(nr)) if nr[s] > j]
        # a batch of the same systems with only right-hand side j
        single = b2s_lib.BatchedCG(off, col, val, rp, ones, tol=1e-10, cluster_size=2)
        Bj = np.zeros(single.vector_length)
        for s in range(len(nr)):
            n = int(rp[s + 1] - rp[s])
            src = Bh[int(multi.vec_off[s]):int(multi.vec_off[s + 1])].reshape(n, int(nr[s]))
            Bj[int(single.vec_off[s]):int(single.vec_off[s + 1])] = src[:, min(j, int(nr[s]) - 1)]
        Bd = cuda.tensor(Bj, device="cuda")
        Xd = cuda.zeros_like(Bd)
        single.solve(Bd, Xd)
        Xj = Xd.cpu().numpy()
        for s in sel:
            n = int(rp[s + 1] - rp[s])
            xm = Xh[int(multi.vec_off[s]):int(multi.vec_off[s + 1])].reshape(n, int(nr[s]))[:, j]
            xs = Xj[int(single.vec_off[s]):int(single.vec_off[s + 1])]
            assert np.array_equal(xm, xs), (s, j)


def test_cluster_sizes_agree_and_autotune(b2s_lib, cuda):
    off, col, val, rp, nr = _batch(nsys=40, seed=6, lo=16, hi=96)
    ref = None
    for c in (1, 2, 4, 8):
        bt = b2s_lib.BatchedCG(off, col, val, rp, nr, tol=1e-11, cluster_size=c)
        B, X = _vectors(cuda, bt, seed=2)
        assert bt.solve(B, X)
        assert bt.report.cluster_size == c
        x = X.cpu().numpy()
        if ref is None:
            ref = x
        else:
            assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) <= 1e-9, c
    bt = b2s_lib.BatchedCG(off, col, val, rp, nr, tol=1e-8)
    B, X = _vectors(cuda, bt, seed=2)
    assert bt.solve(B, X)
    assert bt.report.cluster_size in (1, 2, 4, 8)
    assert bt.report.converged == bt.report.solves == int(nr.sum())
    assert bt.report.max_residue < 1e-8


def test_batch_with_initial_guess_and_unpreconditioned(b2s_lib, cuda):
    off, col, val, rp, nr = _batch(nsys=10, seed=8)
    bt = b2s_lib.BatchedCG(off, col, val, rp, nr, tol=1e-10, preconditioner=None, cluster_size=4)
    B, X = _vectors(cuda, bt, seed=3)
    X.fill_(0.5)
    assert bt.solve(B, X)
    # residual check on the host: ||b - A x|| / ||b|| per right-hand side
    Bh, Xh = B.cpu().numpy(), X.cpu().numpy()
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
    for s in range(len(nr)):
        r0, r1 = int(rp[s]), int(rp[s + 1])
        n, k = r1 - r0, int(nr[s])
        o0, o1 = int(off[r0]), int(off[r1])
        xs = Xh[int(bt.vec_off[s]):int(bt.vec_off[s + 1])].reshape(n, k)
        bs = Bh[int(bt.vec_off[s]):int(bt.vec_off[s + 1])].reshape(n, k)
        ax = np.zeros((n, k))
        np.add.at(ax, rows[o0:o1] - r0, val[o0:o1, None] * xs[col[o0:o1] - r0])
        rel = np.linalg.norm(bs - ax, axis=0) / np.linalg.norm(bs, axis=0)
        assert np.all(rel < 1e-9), (s, rel)
