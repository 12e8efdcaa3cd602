"""The oracle (oracle/b2s_oracle.c, our C restatement of TNL's sparse path)
pinned against (1) the closed-form results of TNL's own SpMV unit tests and
(2) fixtures produced by TNL itself (tests/golden, from oracle/_ref).
CPU only."""
import numpy as np
import pytest

import fixtures as F
import tnl_unit_matrices as U


@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("org", ["col", "row"])
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_tnl_unit_golden_values(oracle, fmt, org, real):
    # SparseMatrixVectorProductTest.hpp: every case has a closed-form result
    for name, (csr, xval, expected) in U.all_cases().items():
        x = np.full(csr[3], xval)
        y = oracle.spmv(fmt, org, csr, x, real=real)
        assert np.array_equal(y, np.asarray(expected, dtype=np.float64)), f"{name} {fmt} {org} {real}"


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("org,real", [("col", "f64"), ("col", "f32"), ("row", "f64")])
def test_layouts_bit_exact_vs_tnl(oracle, name, fmt, org, real):
    got = oracle.convert(fmt, org, F.csr(name), real)
    F.compare_layout(got, F.layout(name, fmt, org, real), fmt)


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_spmv_vs_tnl(oracle, name, fmt, real):
    x, want = F.spmv(name, fmt, real)
    got = oracle.spmv(fmt, "col", F.csr(name), x, real=real)
    scale = max(np.max(np.abs(want)), 1e-300)
    tol = 1e-14 if real == "f64" else 1e-5
    assert np.max(np.abs(got - want)) / scale <= tol


@pytest.mark.parametrize("case", F.solver_cases(), ids=lambda c: c["key"])
def test_solvers_vs_tnl(oracle, case):
    r = oracle.solve(case["solver"], F.csr(case["matrix"]), case["b"], rtol=1e-10, precond=case["precond"],
                     gmres_variant=case["variant"], restart_min=case["restart_min"],
                     restart_max=case["restart_max"], ell=case["ell"])
    assert r["converged"] == case["converged"]
    assert abs(r["iterations"] - case["iterations"]) <= max(2, 0.02 * case["iterations"])
    err = np.max(np.abs(r["x"] - case["x"])) / np.max(np.abs(case["x"]))
    assert err <= 1e-8


def test_keeper_and_row_range(oracle):
    csr = F.csr("irregular_zeros_empty")
    n = len(csr[0]) - 1
    x = np.linspace(-1, 1, csr[3])
    y0 = np.linspace(2, 3, n)
    full = oracle.spmv("csr", "col", csr, x)
    for fmt in F.FORMATS:
        y = oracle.spmv(fmt, "col", csr, x, y0, alpha=2.5, beta=-0.5, begin=10, end=300)
        ref = y0.copy()
        ref[10:300] = -0.5 * y0[10:300] + 2.5 * full[10:300]
        assert np.allclose(y, ref, rtol=1e-14, atol=1e-14)


def test_live_reference_random(oracle):
    """Direct comparison with TNL on fresh random matrices (when the reference build exists)."""
    from oracle import Reference
    try:
        R = Reference()
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built on this machine")
    from b2s import workloads as W
    for seed in range(3):
        csr = W.irregular(1500 + 37 * seed, seed=100 + seed, mu=np.log(8 + 10 * seed), sigma=1.2, hi=700)
        for fmt in F.FORMATS:
            a = oracle.convert(fmt, "col", csr)
            b = R.convert(fmt, "col", csr)
            for k in b:
                assert np.array_equal(a[k], b[k]), (seed, fmt, k)


def _perm_case(seed=7):
    from b2s import workloads as W
    csr = W.irregular(2500, seed=seed, mu=np.log(6), sigma=1.0, hi=180)
    g = np.random.default_rng(seed)
    perm = g.permutation(2500).astype(np.int32)
    return csr, perm, np.argsort(perm).astype(np.int32)


def test_permutations_vs_tnl(oracle):
    """permuteMatrixRows / permuteMatrixColumns / reorderSparseMatrix of the
    oracle against TNL's own functions (oracle/_ref), array for array."""
    from oracle import Reference
    try:
        R = Reference()
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built on this machine")
    csr, perm, iperm = _perm_case()
    a, b = oracle.permute_rows(csr, perm), R.permute_rows(csr, perm)
    assert all(np.array_equal(a[k], b[k]) for k in b)
    # ColumnMajor ChunkedEllpack is excluded: TNL's row view of that layout
    # (ChunkedEllpackSegmentView.h:43-48) addresses offset + local, which is not
    # where the layout stores a row's elements, so TNL maps the wrong slots.
    for fmt in ["csr", "ellpack", "slicedellpack", "biellpack", "slicedellpack16"]:
        a, b = oracle.permute_columns(fmt, "col", csr, iperm), R.permute_columns(fmt, "col", csr, iperm)
        assert all(np.array_equal(a[k], b[k]) for k in b), fmt
    a, b = oracle.reorder(csr, perm, iperm), R.reorder(csr, perm, iperm)
    assert all(np.array_equal(a[k], b[k]) for k in b)


def test_chunked_column_permutation_is_layout_consistent(oracle):
    """ChunkedEllpack: mapping the columns in place equals converting the
    column-mapped CSR matrix (slots keep their order in both)."""
    csr, perm, iperm = _perm_case(11)
    off, col, val, nc = csr
    a = oracle.permute_columns("chunkedellpack", "col", csr, iperm)
    b = oracle.convert("chunkedellpack", "col", (off, iperm[col], val, nc))
    assert all(np.array_equal(a[k], b[k]) for k in b)


@pytest.mark.parametrize("real", ["f64", "f32"])
def test_ilu0_restatement_vs_tnl(oracle, real):
    """The oracle's ILU(0) (factorization + both substitutions) equals TNL's
    Preconditioners::ILU0 update + solve bit for bit."""
    from oracle import Reference
    try:
        ref = Reference()
    except FileNotFoundError:
        pytest.skip("oracle/_ref is not built")
    from b2s import workloads as W
    for csr in (W.convdiff3d(12, seed=4), W.diffusion3d(14, seed=3), W.poisson2d(30), W.laplace3d(9)):
        b = np.random.default_rng(1).uniform(-1, 1, len(csr[0]) - 1)
        assert np.array_equal(oracle.ilu0_apply(csr, b, real), ref.ilu0_apply(csr, b, real))


def _lower_case(n=900, seed=21):
    """A random lower triangle (diagonal included) and its expansion L + L^T - D."""
    g = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        k = int(g.integers(0, min(i, 12) + 1))
        cols = np.sort(np.concatenate([g.choice(i, k, replace=False) if k else np.zeros(0, np.int64), [i]]))
        rows.append(cols)
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    col = np.concatenate(rows).astype(np.int32)
    val = g.normal(size=len(col))
    r_of = np.repeat(np.arange(n), np.diff(off))
    strict = col < r_of
    fr = np.concatenate([r_of, col[strict]])
    fc = np.concatenate([col, r_of[strict]])
    fv = np.concatenate([val, val[strict]])
    order = np.lexsort((fc, fr))
    foff = np.concatenate([[0], np.cumsum(np.bincount(fr, minlength=n))]).astype(np.int32)
    return (off, col, val, n), (foff, fc[order].astype(np.int32), fv[order], n)


def test_symmetric_product_vs_tnl(oracle):
    """SparseMatrix< ..., SymmetricMatrix, CSR >::vectorProduct: the oracle's
    restatement against TNL's own and against the expanded general product."""
    from oracle import Reference
    try:
        R = Reference()
    except FileNotFoundError:
        pytest.skip("oracle/_ref not built on this machine")
    low, full = _lower_case()
    n = low[3]
    x = np.random.default_rng(1).uniform(-1, 1, n)
    y0 = np.random.default_rng(2).uniform(-1, 1, n)
    for alpha, beta, b, e in [(1.0, 0.0, 0, 0), (2.5, -0.5, 0, 0), (1.0, 1.0, 100, 700), (-1.0, 0.25, 899, 900)]:
        got = oracle.spmv_symmetric(low, x, y0, alpha, beta, b, e)
        want = R.spmv_symmetric(low, x, y0, alpha, beta, b, e)
        assert np.max(np.abs(got - want)) <= 1e-13 * max(1.0, np.max(np.abs(want))), (alpha, beta, b, e)
    # the whole range equals the general product of L + L^T - D
    got = oracle.spmv_symmetric(low, x)
    gen = oracle.spmv("csr", "col", full, x)
    assert np.max(np.abs(got - gen)) <= 1e-13 * np.max(np.abs(gen))
