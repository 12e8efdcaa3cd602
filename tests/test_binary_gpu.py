"""Binary matrices: TNL's SparseMatrix< bool, Devices::Cuda, int, ... >
(Matrices/SparseMatrix.h:23-26) through the C ABI (dtype B2S_BOOL).

* layouts: the column indexes and every metadata array equal TNL's own for the
  padded layouts, bit for bit (TNL's binary matrix assigned from the same CSR
  with operator=: capacities from the CSR rows, zero values dropped); a CSR
  binary matrix holds TNL's elements with its -1 slots removed (CSR rows are
  compacted here, as for real matrices); no values are stored;
* the product, bit for bit equal to TNL's host product in ComputeReal = int
  (each stored column adds (int) x[column]; alpha and beta act as ints) for
  FP64 and FP32 vectors, integer-valued and fractional x, the four keepers,
  row ranges, host and device vectors;
* values == NULL stores every entry; solvers and conversion refuse binary
  matrices.
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

LAYOUTS = ["csr", "ellpack", "slicedellpack", "chunkedellpack", "biellpack"]
KEEPERS = [(1.0, 0.0), (2.7, 0.0), (1.0, 0.5), (1.0, 2.0), (-1.5, 3.0), (3.0, -2.25)]


def _binary(b2s, csr, fmt, values=True):
    off, col, val, nc = csr
    return b2s.SparseMatrix.from_csr(off, col, val if values else None, nc, segments=F.SEGMENTS[fmt], real="bool")


def _has_zeros(csr):
    return bool(np.any(np.asarray(csr[2]) == 0))


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("fmt", LAYOUTS)
def test_binary_layout_vs_tnl(b2s_lib, cuda, name, fmt):
    from oracle import Reference
    R = Reference()
    csr = F.csr(name)
    h = R.create(fmt, "col", csr, "bool")
    try:
        want = R.arrays(h)
    finally:
        R.destroy(h)
    M = _binary(b2s_lib, csr, fmt)
    assert len(M.export("values")) == 0
    cols = M.export("columnIndexes")
    if fmt == "csr":
        # TNL keeps a -1 slot for every zero value of the source row
        keep = want["columnIndexes"] != -1
        assert np.array_equal(cols, want["columnIndexes"][keep])
        kept = np.concatenate([[0], np.cumsum(keep.astype(np.int64))])
        wo = kept[want["offsets"]]  # each row's count of non -1 slots, accumulated
        assert np.array_equal(M.export("offsets"), wo)
    else:
        assert np.array_equal(cols, want["columnIndexes"])
        for k, v in want.items():
            if k in ("values", "columnIndexes"):
                continue
            assert np.array_equal(M.export(k), v), k


def _tnl_products(csr, x, real, alpha, beta, y0, begin=0, end=0):
    """TNL's own binary product; the SlicedEllpack matrix is used where TNL's
    CSR would read its -1 slots (a source with zero values)."""
    from oracle import Reference
    R = Reference()
    h = R.create("slicedellpack", "col", csr, "bool")
    try:
        if real == "f64":
            y = np.array(y0, dtype=np.float64, copy=True)
            R._fn("spmv")(h, np.ascontiguousarray(x, np.float64), y, alpha, beta, begin, end)
        else:
            y = np.array(y0, dtype=np.float32, copy=True)
            R.binary_spmv_f32(h, x.astype(np.float32), y, alpha, beta, begin, end)
    finally:
        R.destroy(h)
    return y


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_binary_product_bitwise_vs_tnl(b2s_lib, cuda, name, real):
    csr = F.csr(name)
    n, nc = len(csr[0]) - 1, csr[3]
    dt = np.float64 if real == "f64" else np.float32
    g = np.random.default_rng(7)
    mats = {fmt: _binary(b2s_lib, csr, fmt) for fmt in LAYOUTS}
    for xk, x in (("int", g.integers(-9, 10, nc).astype(dt)), ("frac", g.uniform(-7, 7, nc).astype(dt))):
        y0 = g.uniform(-3, 3, n).astype(dt)
        for alpha, beta in KEEPERS:
            want = _tnl_products(csr, x, real, alpha, beta, y0).astype(dt)
            for fmt, M in mats.items():
                yh = y0.copy()
                M.vectorProduct(x, yh, alpha, beta)  # host vectors
                assert np.array_equal(yh, want), (fmt, xk, alpha, beta)
                yd = cuda.tensor(y0, device="cuda")
                M.vectorProduct(cuda.tensor(x, device="cuda"), yd, alpha, beta)  # device vectors
                assert np.array_equal(yd.cpu().numpy(), want), (fmt, xk, alpha, beta)


@pytest.mark.parametrize("fmt", LAYOUTS)
def test_binary_row_ranges_and_tnl_own_layout(b2s_lib, cuda, fmt):
    from oracle import Reference
    R = Reference()
    for name in F.matrix_names():
        csr = F.csr(name)
        n, nc = len(csr[0]) - 1, csr[3]
        if n < 4:
            continue
        x = np.random.default_rng(3).integers(-4, 5, nc).astype(np.float64)
        y0 = np.linspace(-2, 2, n)
        M = _binary(b2s_lib, csr, fmt)
        b, e = 1, n - 1
        want = _tnl_products(csr, x, "f64", 2.0, 1.0, y0, b, e)
        y = y0.copy()
        M.vectorProduct(x, y, 2.0, 1.0, b, e)
        assert np.array_equal(y, want), name
        if fmt != "csr" or not _has_zeros(csr):
            # TNL's product in the same layout (its CSR only where it has no -1 slots)
            h = R.create(fmt, "col", csr, "bool")
            yt = y0.copy()
            R._fn("spmv")(h, x, yt, 1.0, 0.0, 0, 0)
            R.destroy(h)
            y = y0.copy()
            M.vectorProduct(x, y)
            assert np.array_equal(y, yt), name


def test_binary_without_values_and_refusals(b2s_lib, cuda):
    csr = F.csr(F.matrix_names()[0])
    n, nc = len(csr[0]) - 1, csr[3]
    M = _binary(b2s_lib, csr, "csr", values=False)
    assert np.array_equal(M.export("columnIndexes"), csr[1])  # every entry, zero values too
    y = np.zeros(n)
    M.vectorProduct(np.ones(nc), y)
    assert np.array_equal(y, np.diff(csr[0]).astype(np.float64))  # row lengths
    with pytest.raises(b2s_lib.B2SError) as e:
        s = b2s_lib.CG()
        s.setMatrix(M)
        s.solve(np.ones(n), np.zeros(n))
    assert e.value.status == b2s_lib.UNSUPPORTED
    with pytest.raises(b2s_lib.B2SError) as e:
        M.convert("Ellpack")
    assert e.value.status == b2s_lib.UNSUPPORTED
