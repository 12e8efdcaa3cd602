"""Device assembly (b2s_matrix_from_coo), MatrixMarket input/output and
conversion from padded layouts, on the GPU, against TNL.

* from_coo equals TNL's setRowCapacities( counts ) + setElement / addElement
  (the oracle's restatement, itself pinned to TNL on the CPU) array for array
  in every layout, FP64 and FP32, host and device triplets, with repeated
  pairs and explicit zeros; CSR rows hold exactly the merged elements (TNL's
  CSR keeps an unused -1 slot per merged duplicate);
* the radix-sorted path and the already-sorted fast path give the same
  matrix, and a shuffled 2D Laplacian equals the one built from CSR;
* read_mtx equals TNL's MatrixReader::readMtx, write_mtx writes the bytes of
  TNL's MatrixWriter::writeMtx;
* convert() from every padded layout equals a direct build.
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

LAYOUTS = {"csr": "CSR", "ellpack": "Ellpack", "slicedellpack": "SlicedEllpack", "chunkedellpack": "ChunkedEllpack",
           "biellpack": "BiEllpack", "slicedellpack16": "SlicedEllpack"}
REAL = {"f64": "double", "f32": "float"}


def _compact_csr(a):
    """TNL CSR arrays without the unused (-1) slots."""
    off, col, val = a["offsets"], a["columnIndexes"], a["values"]
    keep = col != -1
    rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
    counts = np.bincount(rows[keep], minlength=len(off) - 1)
    return {"offsets": np.concatenate([[0], np.cumsum(counts)]).astype(np.int64), "columnIndexes": col[keep],
            "values": val[keep]}


def _exports(M, keys):
    return {k: M.export(k) for k in keys}


def _check(M, want, fmt):
    if fmt == "csr":
        want = _compact_csr(want)
    got = _exports(M, want.keys())
    for k in want:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        if k == "values":
            g = g.astype(np.float64)
        assert g.shape == w.shape and np.array_equal(g, w), (fmt, k)


def _triplets(rows, cols, n, seed, zeros=True):
    g = np.random.default_rng(seed)
    ri, ci = g.integers(0, rows, n).astype(np.int32), g.integers(0, cols, n).astype(np.int32)
    v = g.normal(size=n)
    if zeros:
        v[::11] = 0.0
    return ri, ci, v


@pytest.mark.parametrize("fmt", sorted(LAYOUTS))
@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("dup", ["set", "add"])
def test_from_coo_matches_tnl(b2s_lib, cuda, oracle, fmt, real, dup):
    rows, cols = 300, 257
    for seed, n in [(1, 4000), (2, 50), (3, 0)]:
        ri, ci, v = _triplets(rows, cols, n, seed)
        want = oracle.from_coo(fmt, "col", rows, cols, ri, ci, v, dup == "add", real)
        ss = F.SLICE.get(fmt, 0)
        M = b2s_lib.SparseMatrix.from_coo(rows, cols, ri, ci, v, segments=LAYOUTS[fmt], real=REAL[real],
                                          duplicates=dup, slice_size=ss)
        _check(M, want, fmt)
        # the same triplets from device memory
        Md = b2s_lib.SparseMatrix.from_coo(rows, cols, cuda.tensor(ri, device="cuda"), cuda.tensor(ci, device="cuda"),
                                           cuda.tensor(v, device="cuda"), segments=LAYOUTS[fmt], real=REAL[real],
                                           duplicates=dup, slice_size=ss)
        _check(Md, want, fmt)


def test_from_coo_sorted_and_shuffled_agree(b2s_lib, cuda):
    from b2s import workloads as W
    off, col, val, n = W.poisson2d(512)
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(off))
    ref = b2s_lib.SparseMatrix.from_csr(off, col, val, n)
    perm = np.random.default_rng(0).permutation(len(col))
    for order in (np.arange(len(col)), perm):
        M = b2s_lib.SparseMatrix.from_coo(n, n, cuda.tensor(rows[order], device="cuda"),
                                          cuda.tensor(col[order], device="cuda"), cuda.tensor(val[order], device="cuda"))
        for k in ("offsets", "columnIndexes", "values"):
            assert np.array_equal(M.export(k), ref.export(k)), k


def test_from_coo_wide_keys_and_edges(b2s_lib, cuda):
    """Row and column indexes that need 8 radix passes; empty rows; the last
    row and column; repeated pairs summed in input order."""
    rows, cols = (1 << 24) + 3, (1 << 30) + 7
    ri = np.array([rows - 1, 0, 5, rows - 1, 5, 0, 5], np.int32)
    ci = np.array([cols - 1, cols - 1, 3, 0, 3, 0, 3], np.int32)
    v = np.array([1.0, 2.0, 0.1, 4.0, 0.2, 6.0, 0.3])
    M = b2s_lib.SparseMatrix.from_coo(rows, cols, ri, ci, v, duplicates="add")
    off = M.export("offsets")
    assert off[-1] == 5 and off[1] == 2 and off[5] == 2 and off[6] == 3
    assert np.array_equal(M.export("columnIndexes"), [0, cols - 1, 3, 0, cols - 1])
    assert np.array_equal(M.export("values"), [6.0, 2.0, (0.1 + 0.2) + 0.3, 4.0, 1.0])
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.from_coo(4, 4, np.array([0, 4], np.int32), np.array([0, 0], np.int32), np.ones(2))
    assert e.value.status == b2s_lib.INVALID_ARG


@pytest.mark.parametrize("fmt", sorted(LAYOUTS))
def test_read_mtx_matches_tnl(b2s_lib, cuda, oracle, tmp_path, fmt):
    from oracle import Reference
    ref = Reference()
    g = np.random.default_rng(4)
    lines = ["%%MatrixMarket matrix coordinate real symmetric", "% seeded", "90 90 700"]
    for _ in range(700):
        a, b = sorted(g.integers(1, 91, 2))[::-1]
        x = float(g.normal()) if g.random() > 0.05 else 0.0
        lines.append(f"{a} {b} {x!r}")
    p = tmp_path / "s.mtx"
    p.write_text("\n".join(lines) + "\n")
    for real in ("f64", "f32"):
        want = ref.read_mtx(fmt, "col", p, real)
        M = b2s_lib.SparseMatrix.read_mtx(p, segments=LAYOUTS[fmt], real=REAL[real], slice_size=F.SLICE.get(fmt, 0))
        _check(M, want, fmt)


@pytest.mark.parametrize("fmt", sorted(LAYOUTS))
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_write_mtx_matches_tnl_bytes(b2s_lib, cuda, tmp_path, fmt, real):
    from oracle import Reference
    ref = Reference()
    csr = F.csr("irregular_zeros_empty")
    off, col, val, nc = csr
    ours, theirs = tmp_path / "ours.mtx", tmp_path / "tnl.mtx"
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, nc, segments=LAYOUTS[fmt], real=REAL[real],
                                      slice_size=F.SLICE.get(fmt, 0))
    M.write_mtx(ours)
    # TNL's ChunkedEllpack row views do not address the chunk interleave
    # (ChunkedEllpackSegmentView.h:43-48), so its writer prints other rows'
    # slots; the same matrix in Ellpack (zeros dropped alike) is the reference
    ref.write_mtx("ellpack" if fmt == "chunkedellpack" else fmt, "col", csr, theirs, real)
    assert ours.read_bytes() == theirs.read_bytes()


@pytest.mark.parametrize("fmt", [f for f in sorted(LAYOUTS) if f != "csr"])
def test_convert_from_padded_layouts(b2s_lib, cuda, fmt):
    """operator= from a padded layout: TNL takes the capacities from the
    source's non-padding slots and copies the nonzero values."""
    from b2s import workloads as W
    from oracle import Reference
    ref = Reference()
    csr = W.irregular(3000, seed=9, mu=2.0, sigma=1.0, hi=200)
    off, col, val, nc = csr
    val = val.copy()
    val[::7] = 0.0
    csr = (off, col, val, nc)
    P = b2s_lib.SparseMatrix.from_csr(off, col, val, nc, segments=LAYOUTS[fmt], slice_size=F.SLICE.get(fmt, 0))
    for other in ("csr", "ellpack", "slicedellpack", "biellpack", "chunkedellpack"):
        want = ref.assign_to(fmt, "col", csr, other, "col")
        _check(P.convert(LAYOUTS[other]), want, other)
    # a padded source holding explicit zeros (assembled by setElement): the
    # target's capacities count them, the copied elements do not include them
    ri, ci, v = _triplets(200, 150, 3000, 11)
    Z = b2s_lib.SparseMatrix.from_coo(200, 150, ri, ci, v, segments=LAYOUTS[fmt], slice_size=F.SLICE.get(fmt, 0))
    Zc = b2s_lib.SparseMatrix.from_coo(200, 150, ri, ci, v)  # CSR: the merged elements, zeros kept
    zoff, zcol, zval = Zc.export("offsets"), Zc.export("columnIndexes"), Zc.export("values")
    assert np.count_nonzero(zval == 0) > 0
    E = Z.convert("Ellpack")
    if fmt == "ellpack":  # the same type: TNL's copy assignment keeps the triplet-count capacities
        assert np.array_equal(E.export("columnIndexes"), Z.export("columnIndexes"))
        assert np.array_equal(E.export("values"), Z.export("values"))
    else:
        assert E.export("segmentSize")[0] == np.diff(zoff).max()
        assert np.count_nonzero(E.export("columnIndexes") != -1) == np.count_nonzero(zval)
    rows = np.repeat(np.arange(200), np.diff(zoff))
    dense = np.zeros((200, 150))
    np.add.at(dense, (rows, zcol), zval)
    x = np.random.default_rng(2).uniform(-1, 1, 150)
    for other in ("CSR", "Ellpack", "BiEllpack", "ChunkedEllpack"):
        y = np.zeros(200)
        Z.convert(other).vectorProduct(x, y)
        assert np.allclose(y, dense @ x, rtol=1e-12, atol=1e-12), other
