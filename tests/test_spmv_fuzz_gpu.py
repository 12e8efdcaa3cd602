"""Randomized parity of every layout and CSR kernel against the oracle.

Seeded random matrices of edge-case shapes (1-3 rows, counts around the warp,
row-group, row-pair / row-quad and slice boundaries, rectangular both ways)
and row-length profiles (stencil-like, log-normal, mostly empty, one long
row), in FP64 and FP32, with random keepers (alpha, beta) and row ranges,
host and device vectors. The reference is TNL's CSR product restated in the
oracle (b2s_oracle.c) on the same rounded inputs; each row must agree within
the forward error bound of a length-L dot product in the working precision,
|y_i - y_ref_i| <= 2 (L_i + 3) u (|alpha| (|A| |x|)_i + |beta y0_i|), and rows
outside the range must be left bit for bit as they were.
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

REALS = {"f64": ("double", np.float64, 2.0 ** -53), "f32": ("float", np.float32, 2.0 ** -24)}
ROWS = [1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 255, 256, 257, 1023, 1025, 4099]
VARIANTS = [(fmt, {}) for fmt in F.FORMATS] + [
    ("csr", {"csr_row_groups": False}),
    ("csr", {"csr_kernel": "CSRScalar"}),
    ("csr", {"csr_kernel": "CSRVector", "threads_per_row": 4}),
    ("csr", {"csr_kernel": "CSRVector", "threads_per_row": 32}),
]


def _lengths(g, rows, cols, kind):
    if kind == "stencil":
        L = np.full(rows, int(g.integers(3, 10)))
        k = g.choice(rows, size=max(1, rows // 20), replace=False)
        L[k] += g.integers(-2, 3, size=len(k))
    elif kind == "lognormal":
        L = np.rint(np.exp(g.normal(np.log(8.0), 1.2, rows)))
    elif kind == "sparse_rows":
        L = np.where(g.random(rows) < 0.5, 0, g.integers(1, 41, rows))
    else:  # one long row among short ones
        L = np.full(rows, 2)
        L[int(g.integers(0, rows))] = 600
    return np.clip(L, 0, cols).astype(np.int64)


def _matrix(seed):
    g = np.random.default_rng(seed)
    rows = int(ROWS[seed % len(ROWS)])
    cols = int(g.integers(1, 2 * rows + 6))
    kind = ["stencil", "lognormal", "sparse_rows", "long_row"][seed % 4]
    L = _lengths(g, rows, cols, kind)
    off = np.concatenate([[0], np.cumsum(L)]).astype(np.int32)
    col = np.concatenate([np.sort(g.choice(cols, int(l), replace=False)) for l in L] or [[]]).astype(np.int32)
    val = g.normal(size=len(col))
    return (off, col, val, cols), kind


@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("seed", range(16))
def test_random_layouts_kernels_keepers_ranges(b2s_lib, cuda, oracle, seed, real):
    (off, col, val, cols), kind = _matrix(seed)
    rows = len(off) - 1
    rname, dt, u = REALS[real]
    val_r = val.astype(dt).astype(np.float64)  # the matrix as the device stores it
    csr_r = (off, col, val_r, cols)
    g = np.random.default_rng(1000 + seed)
    x = g.uniform(-1, 1, cols).astype(dt)
    y0 = g.uniform(-1, 1, rows).astype(dt)
    lengths = np.diff(off).astype(np.float64)
    row_of = np.repeat(np.arange(rows), np.diff(off))
    absax = np.bincount(row_of, weights=np.abs(val_r) * np.abs(x.astype(np.float64)[col]), minlength=rows)
    cases = [(1.0, 0.0, 0, 0), (float(g.uniform(-2, 2)), float(g.uniform(-2, 2)), 0, 0)]
    b = int(g.integers(0, rows))
    cases.append((float(g.uniform(-2, 2)), float(g.uniform(-2, 2)), b, int(g.integers(b + 1, rows + 1))))
    refs = []
    for alpha, beta, rb, re in cases:
        want = oracle.spmv("csr", "col", csr_r, x.astype(np.float64), y0.astype(np.float64), alpha, beta, rb, re)
        bound = 2.0 * (lengths + 3.0) * u * (abs(alpha) * absax + abs(beta) * np.abs(y0.astype(np.float64)))
        inside = np.zeros(rows, bool)
        inside[rb:(rows if re == 0 else re)] = True
        refs.append((alpha, beta, rb, re, want, bound, inside))
    tdt = cuda.float64 if real == "f64" else cuda.float32
    xd = cuda.tensor(x, dtype=tdt, device="cuda")
    for fmt, kw in VARIANTS:
        M = b2s_lib.SparseMatrix.from_csr(off, col, val, cols, segments=F.SEGMENTS[fmt], real=rname,
                                          slice_size=F.SLICE.get(fmt, 0), **kw)
        for alpha, beta, rb, re, want, bound, inside in refs:
            for where in ("host", "device"):
                if where == "host":
                    y = y0.copy()
                    M.vectorProduct(x, y, alpha, beta, rb, re)
                else:
                    yd = cuda.tensor(y0, dtype=tdt, device="cuda")
                    M.vectorProduct(xd, yd, alpha, beta, rb, re)
                    y = yd.cpu().numpy()
                tag = (seed, kind, rows, cols, fmt, kw, alpha, beta, rb, re, where)
                assert np.array_equal(y[~inside], y0[~inside]), tag
                err = np.abs(y.astype(np.float64) - want)[inside]
                assert np.all(err <= bound[inside] + 1e-300), (tag, float(np.max(err - bound[inside])))


@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("seed", range(8))
def test_random_multidiagonal(b2s_lib, cuda, oracle, seed, real):
    """Multidiagonal matrices of random shape and diagonals (some entries
    absent), random keepers and row ranges: the 16-byte-step and the
    element-wise paths of the product against the oracle's CSR product."""
    g = np.random.default_rng(500 + seed)
    rows = int(ROWS[(3 * seed + 1) % len(ROWS)])
    cols = int(g.integers(1, 2 * rows + 6))
    nd = int(g.integers(1, 12))
    offsets = np.unique(g.integers(-rows + 1, cols, nd))
    R, Cc = [], []
    for o in offsets:
        r = np.arange(max(0, -o), min(rows, cols - o))
        keep = g.random(len(r)) >= 0.15
        R.append(r[keep])
        Cc.append(r[keep] + o)
    R, Cc = np.concatenate(R), np.concatenate(Cc)
    order = np.lexsort((Cc, R))
    R, Cc = R[order], Cc[order]
    off = np.concatenate([[0], np.cumsum(np.bincount(R, minlength=rows))]).astype(np.int32)
    col = Cc.astype(np.int32)
    val = g.normal(size=len(col))
    rname, dt, u = REALS[real]
    val_r = val.astype(dt).astype(np.float64)
    x = g.uniform(-1, 1, cols).astype(dt)
    y0 = g.uniform(-1, 1, rows).astype(dt)
    lengths = np.diff(off).astype(np.float64)
    absax = np.bincount(R, weights=np.abs(val_r) * np.abs(x.astype(np.float64)[col]), minlength=rows)
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, cols, segments="Multidiagonal", real=rname)
    tdt = cuda.float64 if real == "f64" else cuda.float32
    b = int(g.integers(0, rows))
    for alpha, beta, rb, re in [(1.0, 0.0, 0, 0), (float(g.uniform(-2, 2)), float(g.uniform(-2, 2)), b,
                                                   int(g.integers(b + 1, rows + 1)))]:
        want = oracle.spmv("csr", "col", (off, col, val_r, cols), x.astype(np.float64), y0.astype(np.float64),
                           alpha, beta, rb, re)
        bound = 2.0 * (lengths + 3.0) * u * (abs(alpha) * absax + abs(beta) * np.abs(y0.astype(np.float64)))
        inside = np.zeros(rows, bool)
        inside[rb:(rows if re == 0 else re)] = True
        for where in ("host", "device"):
            if where == "host":
                y = y0.copy()
                M.vectorProduct(x, y, alpha, beta, rb, re)
            else:
                yd = cuda.tensor(y0, dtype=tdt, device="cuda")
                M.vectorProduct(cuda.tensor(x, dtype=tdt, device="cuda"), yd, alpha, beta, rb, re)
                y = yd.cpu().numpy()
            tag = (seed, rows, cols, list(offsets), alpha, beta, rb, re, where)
            assert np.array_equal(y[~inside], y0[~inside]), tag
            err = np.abs(y.astype(np.float64) - want)[inside]
            assert np.all(err <= bound[inside] + 1e-300), tag
