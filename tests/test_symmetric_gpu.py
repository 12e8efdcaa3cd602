"""SparseMatrix< Real, Devices::Cuda, int, SymmetricMatrix, Segments > on the
device, in every layout, against TNL's own SymmetricMatrix product
(Devices::Host, compiled from the reference headers; SparseMatrixView.hpp:
413-476).

* the product (atomics, as TNL on the GPU) equals TNL's within 1e-13 (FP64) /
  1e-5 (FP32) relative, for alpha, beta and row ranges, device and host
  vectors, in CSR, Ellpack, SlicedEllpack, ChunkedEllpack and BiEllpack;
* a symmetric matrix in a padded layout stores the lower triangle exactly as
  TNL's layout of that triangle (column indexes and metadata bit for bit);
* assembly from triplets stores (i, j) with i < j at (j, i), as setElement /
  addElement of a SymmetricMatrix do, in every layout; input with an element
  above the diagonal is refused; conversion keeps the matrix symmetric;
* solvers and ILU(0) run on the general form L + L^T - D: bit for bit the
  results of the same matrix given in full, whatever the layout it is stored in;
* operations with no symmetric counterpart here are refused, not approximated.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference()


def _cases():
    import test_oracle as T
    from b2s import workloads as W
    low, full = T._lower_case(3000, seed=5)
    # SPD: the 3D diffusion matrix's lower triangle
    d = W.diffusion3d(14, seed=2)
    off, col, val, n = d
    r_of = np.repeat(np.arange(n), np.diff(off))
    keep = col <= r_of
    loff = np.concatenate([[0], np.cumsum(np.bincount(r_of[keep], minlength=n))]).astype(np.int32)
    return {"random": (low, full), "diffusion": ((loff, col[keep], val[keep], n), d)}


LAYOUTS = ["CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"]
TNL_NAMES = {"Ellpack": "ellpack", "SlicedEllpack": "slicedellpack", "ChunkedEllpack": "chunkedellpack",
             "BiEllpack": "biellpack"}


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("name", ["random", "diffusion"])
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_product_vs_tnl(b2s_lib, cuda, ref, name, real, layout):
    low, full = _cases()[name]
    n = low[3]
    rname, dt, tol = ("double", np.float64, 1e-13) if real == "f64" else ("float", np.float32, 1e-5)
    M = b2s_lib.SparseMatrix.from_csr(*low[:3], n, real=rname, segments=layout, symmetric=True)
    assert M.isSymmetric()
    x = np.random.default_rng(1).uniform(-1, 1, n)
    y0 = np.random.default_rng(2).uniform(-1, 1, n)
    for alpha, beta, b, e in [(1.0, 0.0, 0, 0), (2.5, -0.5, 0, 0), (1.0, 1.0, 100, n - 300), (-1.0, 0.25, n - 1, n)]:
        want = ref.spmv_symmetric(low, x, y0, alpha, beta, b, e, real=real)
        scale = max(1.0, np.max(np.abs(want)))
        yh = y0.astype(dt).copy()
        M.vectorProduct(x.astype(dt), yh, alpha, beta, b, e)
        assert np.max(np.abs(yh - want)) <= tol * scale, (alpha, beta, b, e, "host")
        tdt = cuda.float64 if real == "f64" else cuda.float32
        yd = cuda.tensor(y0, dtype=tdt, device="cuda")
        M.vectorProduct(cuda.tensor(x, dtype=tdt, device="cuda"), yd, alpha, beta, b, e)
        assert np.max(np.abs(yd.cpu().numpy() - want)) <= tol * scale, (alpha, beta, b, e, "device")
    # the arrays are stored as given: the lower triangle, in TNL's layout of it
    if layout == "CSR":
        assert np.array_equal(M.export("columnIndexes"), low[1])
    else:
        h = ref.create(TNL_NAMES[layout], "col", low)
        try:
            want = ref.arrays(h)
        finally:
            ref.destroy(h)
        for k, v in want.items():
            if k != "values":
                assert np.array_equal(M.export(k), v), k


def test_assembly_and_refusals(b2s_lib, cuda):
    low, full = _cases()["random"]
    off, col, val, n = low
    r_of = np.repeat(np.arange(n), np.diff(off))
    g = np.random.default_rng(3)
    # every element given at (i, j) or (j, i) at random, in shuffled order
    flip = g.random(len(col)) < 0.5
    ri = np.where(flip, col, r_of).astype(np.int32)
    ci = np.where(flip, r_of, col).astype(np.int32)
    order = g.permutation(len(col))
    A = b2s_lib.SparseMatrix.from_coo(n, n, ri[order], ci[order], val[order], symmetric=True)
    assert A.isSymmetric()
    assert np.array_equal(A.export("columnIndexes"), col) and np.array_equal(A.export("values"), val)
    # addElement of a mirrored duplicate adds into the stored element
    ra = np.concatenate([ri, ci]).astype(np.int32)
    ca = np.concatenate([ci, ri]).astype(np.int32)
    va = np.concatenate([val, val])
    B = b2s_lib.SparseMatrix.from_coo(n, n, ra, ca, va, symmetric=True, duplicates="add")
    assert np.array_equal(B.export("values"), 2 * val)
    # the same triplets assembled into the padded layouts: the lower triangle in each
    x = np.random.default_rng(8).uniform(-1, 1, n)
    yc = np.zeros(n)
    A.vectorProduct(x, yc)
    for layout in LAYOUTS[1:]:
        P = b2s_lib.SparseMatrix.from_coo(n, n, ri[order], ci[order], val[order], segments=layout, symmetric=True)
        assert P.isSymmetric()
        y = np.zeros(n)
        P.vectorProduct(x, y)
        assert np.max(np.abs(y - yc)) <= 1e-13 * np.max(np.abs(yc)), layout
    # refusals: an element above the diagonal, in CSR and in a padded layout
    k = int(np.flatnonzero(np.diff(off) > 1)[0])  # a row with an element left of the diagonal
    up_col = col.copy()
    up_col[off[k]] = k + 1
    for layout in ("CSR", "SlicedEllpack"):
        with pytest.raises(b2s_lib.B2SError) as e:
            b2s_lib.SparseMatrix.from_csr(off, up_col, val, n, segments=layout, symmetric=True)
        assert e.value.status == b2s_lib.INVALID_ARG
    # conversions keep a SymmetricMatrix one: CSR -> padded -> padded -> CSR
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, n, symmetric=True)
    S = M.convert("SlicedEllpack")
    B = S.convert("BiEllpack", "float")
    C = B.convert("CSR", "double")
    for T in (S, B, C, M.convert("CSR", "float")):
        assert T.isSymmetric()
    assert np.array_equal(C.export("columnIndexes"), col)
    assert np.array_equal(C.export("values"), val.astype(np.float32).astype(np.float64))


@pytest.mark.parametrize("layout", ["CSR", "SlicedEllpack", "ChunkedEllpack"])
@pytest.mark.parametrize("kind,pre", [("cg", None), ("cg", "diagonal"), ("cg", "ilu0"), ("gmres", "ilu0")])
def test_solvers_on_the_general_form(b2s_lib, cuda, kind, pre, layout):
    low, full = _cases()["diffusion"]
    n = low[3]
    b = np.random.default_rng(4).uniform(-1, 1, n)
    out = []
    for csr, sym, seg in ((low, True, layout), (full, False, "CSR")):
        M = b2s_lib.SparseMatrix.from_csr(*csr[:3], n, segments=seg, symmetric=sym)
        s = {"cg": b2s_lib.CG, "gmres": b2s_lib.GMRES}[kind]()
        s.setMatrix(M)
        s.setPreconditioner(pre)
        s.setConvergenceResidue(1e-10)
        x = np.zeros(n)
        assert s.solve(b, x)
        out.append((s.getIterations(), x))
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    # the stand-alone preconditioner too
    Ms = b2s_lib.SparseMatrix.from_csr(*low[:3], n, segments=layout, symmetric=True)
    Mf = b2s_lib.SparseMatrix.from_csr(*full[:3], n)
    z1, z2 = np.zeros(n), np.zeros(n)
    b2s_lib.Preconditioner(Ms, "ilu0").solve(b, z1)
    b2s_lib.Preconditioner(Mf, "ilu0").solve(b, z2)
    assert np.array_equal(z1, z2)
