"""Matrices::MultidiagonalMatrix on the device against TNL's own
(Devices::Host, compiled from the reference headers;
MultidiagonalMatrixView.hpp:488-528), through the C ABI.

* layout: the diagonals are the pattern's distinct (column - row) offsets,
  ascending; the values array equals TNL's ColumnMajor MultidiagonalMatrix
  (the Devices::Cuda organization) built with the same offsets and elements,
  bit for bit, FP64 and FP32, square and rectangular, with empty rows;
* product: TNL's keepers (alpha, beta), row ranges, host and device vectors,
  within 1e-14 (FP64) / 1e-6 (FP32) relative of TNL's product;
* the solvers run on it as on the sparse layouts: CG, BiCGStab, GMRES, TFQMR
  reach the CSR matrix's iterates in as many iterations; mixed precision
  converges to the FP64 tolerance; conversions to and from CSR keep the
  elements;
* refused: more than 128 diagonals, binary and symmetric matrices, column
  permutation, binary files.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference()


def _band(rows, cols, offsets, seed, drop=0.0):
    """A rows x cols matrix on the given diagonals, some entries absent."""
    g = np.random.default_rng(seed)
    R, Cc, V = [], [], []
    for r in range(rows):
        for o in offsets:
            c = r + o
            if 0 <= c < cols and g.random() >= drop:
                R.append(r)
                Cc.append(c)
                V.append(g.normal() + (4.0 if o == 0 else 0.0))
    R, Cc, V = np.array(R), np.array(Cc), np.array(V)
    off = np.concatenate([[0], np.cumsum(np.bincount(R, minlength=rows))]).astype(np.int32)
    return off, Cc.astype(np.int32), V, cols


def _matrices():
    from b2s import workloads as W
    return {"laplace3d": W.laplace3d(9), "convdiff": W.convdiff3d(7, seed=3), "poisson": W.poisson2d(17),
            "band_tall": _band(60, 40, [-7, -2, 0, 3], 1, drop=0.2),
            "band_wide": _band(35, 70, [-3, 0, 1, 5, 30], 2, drop=0.3)}


def _dense_rows(csr, offsets):
    """values[r, d] = A(r, r + offsets[d]) (0 where absent)."""
    off, col, val, nc = csr
    n = len(off) - 1
    idx = {o: d for d, o in enumerate(offsets)}
    out = np.zeros((n, len(offsets)))
    for r in range(n):
        for k in range(off[r], off[r + 1]):
            out[r, idx[col[k] - r]] = val[k]
    return out


@pytest.mark.parametrize("name", list(_matrices()))
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_layout_and_product_vs_tnl(b2s_lib, cuda, ref, name, real):
    csr = _matrices()[name]
    off, col, val, nc = csr
    n = len(off) - 1
    rname = "double" if real == "f64" else "float"
    dt = np.float64 if real == "f64" else np.float32
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, nc, segments="Multidiagonal", real=rname)
    rows = np.repeat(np.arange(n), np.diff(off))
    want_offsets = np.unique(col.astype(np.int64) - rows)
    got_offsets = M.export("diagonalsOffsets")
    assert np.array_equal(got_offsets, want_offsets)
    h = ref.multidiagonal(n, nc, want_offsets, _dense_rows(csr, want_offsets), real=real)
    try:
        want_vals = ref.mdiag_values(h)
        assert np.array_equal(M.export("values").astype(np.float64), want_vals)
        g = np.random.default_rng(4)
        x = g.uniform(-1, 1, nc).astype(dt).astype(np.float64)
        y0 = g.uniform(-1, 1, n).astype(dt).astype(np.float64)
        tol = 1e-14 if real == "f64" else 1e-6
        for alpha, beta, b, e in [(1.0, 0.0, 0, 0), (2.0, -0.5, 0, 0), (1.0, 1.0, 3, n - 5), (-1.5, 0.0, 1, n)]:
            want = ref.mdiag_spmv(h, x, y0, alpha, beta, b, e)
            scale = max(1.0, np.max(np.abs(want)))
            yh = y0.astype(dt).copy()
            M.vectorProduct(x.astype(dt), yh, alpha, beta, b, e)
            assert np.max(np.abs(yh - want)) <= tol * scale, (alpha, beta, b, e)
            tdt = cuda.float64 if real == "f64" else cuda.float32
            yd = cuda.tensor(y0, dtype=tdt, device="cuda")
            M.vectorProduct(cuda.tensor(x, dtype=tdt, device="cuda"), yd, alpha, beta, b, e)
            assert np.max(np.abs(yd.cpu().numpy() - want)) <= tol * scale
    finally:
        ref.mdiag_destroy(h)


def test_conversions_keep_the_elements(b2s_lib, cuda):
    for name, csr in _matrices().items():
        off, col, val, nc = csr
        M = b2s_lib.SparseMatrix.from_csr(off, col, val, nc, segments="Multidiagonal")
        C = M.convert("CSR")  # zeros of absent diagonal entries are not copied
        assert np.array_equal(C.export("offsets"), off), name
        assert np.array_equal(C.export("columnIndexes"), col), name
        assert np.array_equal(C.export("values"), val), name
        S = b2s_lib.SparseMatrix.from_csr(off, col, val, nc).convert("Multidiagonal", "float")
        assert np.array_equal(S.export("values"), M.export("values").astype(np.float32)), name


@pytest.mark.parametrize("kind,name", [("CG", "poisson"), ("BICGStab", "convdiff"), ("GMRES", "convdiff"),
                                       ("TFQMR", "convdiff")])
@pytest.mark.parametrize("pre", [None, "diagonal"])
def test_solvers_equal_the_csr_iterates(b2s_lib, cuda, kind, name, pre):
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(5).uniform(-1, 1, n)
    out = []
    for seg in ("CSR", "Multidiagonal"):
        M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=seg)
        s = getattr(b2s_lib, kind)()
        s.setMatrix(M)
        s.setPreconditioner(pre)
        s.setConvergenceResidue(1e-10)
        x = np.zeros(n)
        assert s.solve(b, x)
        out.append((s.getIterations(), x))
    assert out[0][0] == out[1][0]
    assert np.max(np.abs(out[0][1] - out[1][1])) <= 1e-13 * np.max(np.abs(out[0][1]))


@pytest.mark.parametrize("kind", ["CG", "BICGStab", "GMRES"])
def test_mixed_precision(b2s_lib, cuda, kind):
    csr = _matrices()["poisson" if kind == "CG" else "convdiff"]
    n = len(csr[0]) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments="Multidiagonal", keep_fp32_copy=True)
    s = getattr(b2s_lib, kind)()
    s.setMatrix(M)
    s.setConvergenceResidue(1e-10)
    s.setPrecision(True)
    x = np.zeros(n)
    assert s.solve(b, x)
    assert s.report.true_residual <= 1e-10
    F = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = getattr(b2s_lib, kind)()
    s.setMatrix(F)
    s.setConvergenceResidue(1e-12)
    x64 = np.zeros(n)
    assert s.solve(b, x64)
    assert np.max(np.abs(x - x64)) <= 1e-7 * np.max(np.abs(x64))


def test_refusals(b2s_lib, cuda, tmp_path):
    from b2s import workloads as W
    irr = W.irregular(3000, seed=2, mu=np.log(8), sigma=1.0, hi=200)
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.from_csr(*irr[:3], irr[3], segments="Multidiagonal")
    assert e.value.status == b2s_lib.UNSUPPORTED
    csr = _matrices()["poisson"]
    for kw in ({"real": "bool"}, {"symmetric": True}):
        with pytest.raises(b2s_lib.B2SError) as e:
            b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments="Multidiagonal", **kw)
        assert e.value.status == b2s_lib.UNSUPPORTED
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments="Multidiagonal")
    with pytest.raises(b2s_lib.B2SError) as e:
        M.permuteColumns(np.arange(csr[3], dtype=np.int32))
    assert e.value.status == b2s_lib.UNSUPPORTED
    with pytest.raises(b2s_lib.B2SError) as e:
        M.save(str(tmp_path / "m.tnl"))
    assert e.value.status == b2s_lib.UNSUPPORTED


def test_autotuner_considers_it(b2s_lib, cuda):
    from b2s import workloads as W
    csr = W.laplace3d(40)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    best, table = b2s_lib.autotune(M, reps=3)
    md = [t for t in table if t["segments"] == "Multidiagonal"]
    assert len(md) == 1 and not md[0]["skipped"]


def test_from_offsets_and_values(b2s_lib, cuda, ref):
    """SparseMatrix.multidiagonal: TNL's setDimensions( rows, cols, offsets ) + setElement."""
    g = np.random.default_rng(9)
    rows, cols, offsets = 50, 45, [4, -6, 0, -1]
    vals = g.normal(size=(rows, len(offsets)))
    M = b2s_lib.SparseMatrix.multidiagonal(rows, cols, offsets, vals)
    srt = np.argsort(offsets)
    assert np.array_equal(M.export("diagonalsOffsets"), np.sort(offsets))
    h = ref.multidiagonal(rows, cols, np.sort(offsets), vals[:, srt])
    try:
        assert np.array_equal(M.export("values"), ref.mdiag_values(h))
        x = g.uniform(-1, 1, cols)
        y = np.zeros(rows)
        M.vectorProduct(x, y)
        want = ref.mdiag_spmv(h, x, np.zeros(rows))
        assert np.max(np.abs(y - want)) <= 1e-14 * np.max(np.abs(want))
    finally:
        ref.mdiag_destroy(h)


@pytest.mark.parametrize("real", ["double", "float"])
def test_empty_and_degenerate(b2s_lib, cuda, real):
    """0 x 0, rows without elements, 1 x 1, and a tall matrix whose lowest
    diagonal reaches past the square part (TNL's element count per diagonal
    is min(rows, cols - offsets[0]) then): the product against a dense one."""
    dt = np.float64 if real == "double" else np.float32
    M = b2s_lib.SparseMatrix.from_csr(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0,
                                      segments="Multidiagonal", real=real)
    M.vectorProduct(np.zeros(0, dt), np.zeros(0, dt))
    M = b2s_lib.SparseMatrix.from_csr(np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0), 4,
                                      segments="Multidiagonal", real=real)
    y = np.full(5, 7.0, dt)
    M.vectorProduct(np.ones(4, dt), y)
    assert np.array_equal(y, np.zeros(5, dt))
    for csr in [(np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.5]), 1),
                _band(10, 3, [-7, 0], 5), _band(9, 5, [-8, -3, 1], 6, drop=0.2)]:
        off, col, val, nc = csr
        n = len(off) - 1
        M = b2s_lib.SparseMatrix.from_csr(off, col, val, nc, segments="Multidiagonal", real=real)
        dense = np.zeros((n, nc))
        dense[np.repeat(np.arange(n), np.diff(off)), col] = val.astype(dt)
        x = np.random.default_rng(n).uniform(-1, 1, nc).astype(dt)
        want = dense @ x.astype(np.float64)
        for vec in ("host", "device"):
            if vec == "host":
                y = np.full(n, 3.0, dt)
                M.vectorProduct(x, y)
            else:
                tdt = cuda.float64 if real == "double" else cuda.float32
                yd = cuda.full((n,), 3.0, dtype=tdt, device="cuda")
                M.vectorProduct(cuda.tensor(x, device="cuda"), yd)
                y = yd.cpu().numpy()
            tol = 1e-14 if real == "double" else 1e-6
            assert np.max(np.abs(y - want)) <= tol * max(1.0, np.max(np.abs(want))), (n, nc, vec)
