"""Row / column permutations and reordering on the device
(Matrices/MatrixPermutationApplier.h, Matrices/SparseOperations.h) against the
oracle, which is pinned to TNL's own functions in test_oracle.py: storage
arrays bit-exact."""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu


def _case(seed=5, rows=3000):
    from b2s import workloads as W
    csr = W.irregular(rows, seed=seed, mu=np.log(7), sigma=1.1, hi=300)
    g = np.random.default_rng(seed)
    perm = g.permutation(rows).astype(np.int32)
    return csr, perm, np.argsort(perm).astype(np.int32)


def _arrays(M, keys):
    return {k: M.export(k) for k in keys}


def test_permute_rows_csr(b2s_lib, cuda, oracle):
    csr, perm, _ = _case()
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    M.permuteRows(perm)
    want = oracle.permute_rows(csr, perm)
    F.compare_layout(_arrays(M, want.keys()), want, "csr")
    # the product follows: (P A) x = P (A x)
    x = np.random.default_rng(1).uniform(-1, 1, csr[3])
    y = np.zeros(len(perm))
    M.vectorProduct(x, y)
    ref = oracle.spmv("csr", "col", csr, x)[perm]
    assert np.max(np.abs(y - ref)) / np.max(np.abs(ref)) <= 1e-12


@pytest.mark.parametrize("fmt", F.FORMATS)
def test_permute_columns_every_layout(b2s_lib, cuda, oracle, fmt):
    csr, _, iperm = _case(6)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=F.SEGMENTS[fmt], slice_size=F.SLICE.get(fmt, 0))
    M.permuteColumns(cuda.tensor(iperm, device="cuda"))
    want = oracle.permute_columns(fmt, "col", csr, iperm)
    F.compare_layout(_arrays(M, want.keys()), want, fmt)


def test_reorder_and_symmetric_permutation_solve(b2s_lib, cuda, oracle):
    from b2s import workloads as W
    csr = W.diffusion3d(14, seed=2)
    n = len(csr[0]) - 1
    g = np.random.default_rng(3)
    perm = g.permutation(n).astype(np.int32)
    iperm = np.argsort(perm).astype(np.int32)
    A = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    B = A.reorder(perm, iperm)
    want = oracle.reorder(csr, perm, iperm)
    F.compare_layout(_arrays(B, want.keys()), want, "csr")
    # the same symmetric permutation in place (rows, then columns; unsorted rows)
    A.permuteRows(perm)
    A.permuteColumns(iperm)
    b = W.uniform(n, 4)
    xs = []
    for M, rhs in ((b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3]), b), (B, b[perm]), (A, b[perm])):
        s = b2s_lib.CG()
        s.setMatrix(M)
        s.setPreconditioner("diagonal")  # the diagonal must follow the permutation
        s.setConvergenceResidue(1e-11)
        x = np.zeros(n)
        assert s.solve(rhs, x)
        xs.append(x)
    for x in xs[1:]:
        assert np.max(np.abs(x - xs[0][perm])) / np.max(np.abs(xs[0])) <= 1e-8


def test_reorder_array_and_bad_permutations(b2s_lib, cuda):
    g = np.random.default_rng(9)
    perm = cuda.tensor(g.permutation(10007).astype(np.int32), device="cuda")
    for dt in (cuda.float64, cuda.float32, cuda.int32):
        src = cuda.arange(10007, device="cuda").to(dt)
        dst = cuda.empty_like(src)
        b2s_lib.reorderArray(src, dst, perm)
        assert cuda.equal(dst, src[perm.long()])
    csr, p, _ = _case(8, rows=500)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    bad = p.copy()
    bad[17] = 500
    with pytest.raises(b2s_lib.B2SError):
        M.permuteRows(bad)
    S = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments="SlicedEllpack")
    with pytest.raises(b2s_lib.B2SError):
        S.permuteRows(p)  # rows of padded layouts: permute the CSR matrix, then convert
