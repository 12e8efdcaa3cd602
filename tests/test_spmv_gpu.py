"""GPU parity of the segment layouts and SpMV (through the C ABI).

* layouts: bit-exact against TNL's own arrays (tests/golden) and the oracle
* SpMV: FP64 within 1e-12 relative (max |y - y_ref| / max |y_ref|) of TNL's
  Devices::Host result; FP32 within 1e-5 relative of TNL's FP32 result;
  closed-form golden values of TNL's unit tests exactly
"""
import numpy as np
import pytest

import fixtures as F
import tnl_unit_matrices as U

pytestmark = pytest.mark.gpu

REALS = {"f64": ("double", np.float64), "f32": ("float", np.float32)}


def make(b2s, csr, fmt, real="f64", **kw):
    off, col, val, nc = csr
    return b2s.SparseMatrix.from_csr(off, col, val, nc, segments=F.SEGMENTS[fmt], real=REALS[real][0],
                                     slice_size=F.SLICE.get(fmt, 0), **kw)


def export_all(M, want_keys):
    return {k: M.export(k) for k in want_keys}


def rel_err(got, want):
    return np.max(np.abs(got - want)) / max(np.max(np.abs(want)), 1e-300) if len(want) else 0.0


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_layout_bit_exact_vs_tnl(b2s_lib, cuda, name, fmt, real):
    want = F.layout(name, fmt, "col", real)
    M = make(b2s_lib, F.csr(name), fmt, real)
    got = export_all(M, want.keys())
    F.compare_layout(got, want, fmt)


@pytest.mark.parametrize("name", F.matrix_names())
@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_spmv_vs_tnl(b2s_lib, cuda, name, fmt, real):
    x, want = F.spmv(name, fmt, real)
    M = make(b2s_lib, F.csr(name), fmt, real)
    dt = cuda.float64 if real == "f64" else cuda.float32
    xd = cuda.tensor(x, dtype=dt, device="cuda")
    yd = cuda.zeros(len(want), dtype=dt, device="cuda")
    M.vectorProduct(xd, yd)
    got = yd.cpu().numpy().astype(np.float64)
    assert rel_err(got, want) <= (1e-12 if real == "f64" else 1e-5)


@pytest.mark.parametrize("fmt", F.FORMATS)
@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("kernel,tpr", [("CSRDefault", 0), ("CSRScalar", 0), ("CSRVector", 2), ("CSRVector", 32)])
def test_tnl_unit_golden_values(b2s_lib, cuda, fmt, real, kernel, tpr):
    if fmt != "csr" and kernel != "CSRDefault":
        pytest.skip("CSR kernel choice applies to CSR only")
    dt = REALS[real][1]
    for name, (csr, xval, expected) in U.all_cases().items():
        M = make(b2s_lib, csr, fmt, real, csr_kernel=kernel, threads_per_row=tpr)
        x = np.full(csr[3], xval, dtype=dt)
        y = np.zeros(len(csr[0]) - 1, dtype=dt)
        M.vectorProduct(x, y)  # host vectors through the ABI
        assert np.array_equal(y.astype(np.float64), np.asarray(expected, np.float64)), name


@pytest.mark.parametrize("fmt", F.FORMATS)
def test_keepers_and_row_ranges(b2s_lib, cuda, oracle, fmt):
    csr = F.csr("irregular_zeros_empty")
    n = len(csr[0]) - 1
    x = np.linspace(-1, 1, csr[3])
    y0 = np.linspace(2, 3, n)
    M = make(b2s_lib, csr, fmt)
    for alpha, beta, b, e in [(1, 0, 0, 0), (2.5, 0, 0, 0), (1, 0.5, 0, 0), (-1.5, 2.0, 3, n - 3), (1, 0, 17, 18),
                              (1, 0, 0, 1), (0.0, 1.0, 0, 0)]:
        y = y0.copy()
        M.vectorProduct(x, y, alpha, beta, b, e)
        ref = oracle.spmv(fmt, "col", csr, x, y0, alpha, beta, b, e)
        assert rel_err(y, ref) <= 1e-13, (alpha, beta, b, e)


@pytest.mark.parametrize("fmt", F.FORMATS)
def test_host_and_device_vectors_agree(b2s_lib, cuda, fmt):
    csr = F.csr("irregular_long")
    M = make(b2s_lib, csr, fmt)
    x = np.random.default_rng(0).uniform(-1, 1, csr[3])
    yh = np.zeros(len(csr[0]) - 1)
    M.vectorProduct(x, yh)
    xd = cuda.tensor(x, device="cuda")
    yd = cuda.zeros(len(yh), dtype=cuda.float64, device="cuda")
    M.vectorProduct(xd, yd)
    assert np.array_equal(yd.cpu().numpy(), yh)  # same kernel, same order: identical bits


def test_pipelined_host_vectors(b2s_lib, cuda):
    """Host vectors on a large CSR matrix with short rows go up and down in
    chunks overlapped with the chunked products: the result equals the
    device-vector product bit for bit — banded and random columns, a
    rectangular matrix, trailing empty rows, alpha != 1, repeated calls, FP32;
    matrices with long rows take the unchunked path, also bit for bit."""
    from b2s import workloads as W
    g = np.random.default_rng(3)
    lap = W.laplace3d(48)
    irr = W.irregular(150000, seed=4, mu=1.0, sigma=0.5, hi=7)
    n = 90000  # rectangular, 3 x more columns, the last 1000 rows empty
    lens = np.concatenate([g.integers(0, 9, n - 1000), np.zeros(1000, np.int64)])
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(g.choice(3 * n, L, replace=False)) for L in lens]).astype(np.int32)
    rect = (off, col, g.normal(size=len(col)), 3 * n)
    long = W.irregular(100000, seed=5, mu=2.0, sigma=1.0, hi=600)
    for name, csr in (("laplace", lap), ("irregular", irr), ("rectangular", rect), ("long_rows", long)):
        for real, dt in (("double", np.float64), ("float", np.float32)):
            M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], real=real)
            x = g.uniform(-1, 1, csr[3]).astype(dt)
            tdt = cuda.float64 if dt == np.float64 else cuda.float32
            for alpha in (1.0, -2.5):
                yd = cuda.empty(len(csr[0]) - 1, dtype=tdt, device="cuda")
                M.vectorProduct(cuda.tensor(x, device="cuda"), yd, alpha)
                want = yd.cpu().numpy()
                for _ in range(2):
                    yh = np.full(len(csr[0]) - 1, 7.0, dtype=dt)
                    M.vectorProduct(x, yh, alpha)
                    assert np.array_equal(yh, want), (name, real, alpha)
                # page-locked vectors: the pipeline replayed as one graph (rebuilt for a new alpha)
                xp = cuda.tensor(x).pin_memory()
                yp = cuda.full((len(csr[0]) - 1,), 7.0, dtype=tdt).pin_memory()
                for _ in range(3):
                    yp.fill_(7.0)
                    M.vectorProduct(xp.numpy(), yp.numpy(), alpha)
                    assert np.array_equal(yp.numpy(), want), (name, real, alpha, "pinned")


@pytest.mark.parametrize("fmt", F.FORMATS)
def test_random_matrices_vs_oracle(b2s_lib, cuda, oracle, fmt):
    from b2s import workloads as W
    for seed, rows, mu, hi in [(11, 5000, 2.0, 300), (12, 20001, 3.0, 2048), (13, 777, 0.5, 40)]:
        csr = W.irregular(rows, seed=seed, mu=mu, sigma=1.3, hi=hi)
        want = oracle.convert(fmt, "col", csr)
        M = make(b2s_lib, csr, fmt)
        F.compare_layout(export_all(M, want.keys()), want, fmt)
        x = W.uniform(csr[3], seed)
        y = np.zeros(rows)
        M.vectorProduct(x, y)
        assert rel_err(y, oracle.spmv(fmt, "col", csr, x)) <= 1e-12


def _rows_csr(lengths, ncols, seed):
    g = np.random.default_rng(seed)
    off = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int32)
    col = np.concatenate([np.sort(g.choice(ncols, L, replace=False)) for L in lengths] or [[]]).astype(np.int32)
    return off, col, g.normal(size=len(col)), ncols


@pytest.mark.parametrize("real", ["f64", "f32"])
def test_csr_row_groups_and_windows(b2s_lib, cuda, oracle, real):
    """The adaptive CSR path runs 32-row groups staged in shared memory when
    every group holds <= 256 nonzeros, nnz windows otherwise: both agree with
    TNL, at the cap, one past it, with ragged tails, empty rows and a single
    long row filling a group."""
    cases = {
        "stencil_ragged": ([7] * 1000 + [3, 0, 5], True),
        "cap_exact": ([8] * 64 + [0] * 31 + [256] + [1] * 7, True),
        "cap_plus_one": ([8] * 31 + [9] + [8] * 40, False),
        "long_row": ([2] * 40 + [600] + [2] * 40, False),
        "empty_rows": ([0] * 70 + [5] * 33 + [0] * 3, True),
    }
    tol = 1e-12 if real == "f64" else 1e-5
    for name, (lengths, groups) in cases.items():
        csr = _rows_csr(lengths, 700, len(lengths))
        x = np.random.default_rng(1).uniform(-1, 1, csr[3])
        ref = oracle.spmv("csr", "col", csr, x)
        for allow in (True, False):
            M = make(b2s_lib, csr, "csr", real, csr_row_groups=allow)
            assert M.info.csr_path == (1 if groups and allow else 2), name
            yh = np.zeros(len(lengths), dtype=REALS[real][1])
            M.vectorProduct(x.astype(REALS[real][1]), yh)
            assert rel_err(yh.astype(np.float64), ref) <= tol, (name, allow)
            yd = cuda.zeros(len(lengths), dtype=cuda.float64 if real == "f64" else cuda.float32, device="cuda")
            M.vectorProduct(cuda.tensor(x, dtype=yd.dtype, device="cuda"), yd)
            assert rel_err(yd.cpu().numpy().astype(np.float64), ref) <= tol, (name, allow)


def test_empty_and_degenerate(b2s_lib, cuda):
    for fmt in F.FORMATS:
        # 0 x 0
        M = make(b2s_lib, (np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0), fmt)
        M.vectorProduct(np.zeros(0), np.zeros(0))
        # rows without any element
        csr = (np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0), 4)
        M = make(b2s_lib, csr, fmt)
        y = np.full(5, 7.0)
        M.vectorProduct(np.ones(4), y)
        assert np.array_equal(y, np.zeros(5))


def test_invalid_inputs_are_rejected(b2s_lib, cuda):
    bad_cols = (np.array([0, 2], np.int32), np.array([0, 5], np.int32), np.array([1.0, 2.0]), 3)
    with pytest.raises(b2s_lib.B2SError) as e:
        make(b2s_lib, bad_cols, "csr")
    assert e.value.status == b2s_lib.INVALID_ARG
    bad_off = (np.array([0, 3, 2], np.int32), np.array([0, 1, 2], np.int32), np.ones(3), 3)
    with pytest.raises(b2s_lib.B2SError):
        make(b2s_lib, bad_off, "ellpack")


def test_full_size_laplace3d_properties(b2s_lib, cuda):
    """128^3 7-point Laplacian (2.1M rows, 14.6M nnz): A*1 gives the exact row
    sums, all layouts agree bit for bit with CSR, and SpMV is linear."""
    from b2s import workloads as W
    csr = W.laplace3d(128)
    n = len(csr[0]) - 1
    rows = np.repeat(np.arange(n), np.diff(csr[0]))
    rowsum = np.bincount(rows, weights=csr[2], minlength=n)
    ones = cuda.ones(n, dtype=cuda.float64, device="cuda")
    x = cuda.tensor(W.uniform(n, 1), device="cuda")
    y_ref = None
    for fmt in F.FORMATS:
        M = make(b2s_lib, csr, fmt)
        y = cuda.empty(n, dtype=cuda.float64, device="cuda")
        M.vectorProduct(ones, y)
        assert np.array_equal(y.cpu().numpy(), rowsum), fmt
        M.vectorProduct(x, y)
        if y_ref is None:
            y_ref = y.clone()
        else:
            assert float((y - y_ref).abs().max() / y_ref.abs().max()) <= 1e-14, fmt
        y2 = cuda.empty_like(y)
        M.vectorProduct(2.0 * x + ones, y2)
        lin = 2.0 * y + cuda.tensor(rowsum, device="cuda")
        assert float((y2 - lin).abs().max() / lin.abs().max()) <= 1e-13
