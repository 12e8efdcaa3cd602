"""TNL's binary matrix files (SparseMatrix::save / load) against TNL itself.

* a file written here is byte for byte the file TNL writes for the same
  matrix (the unused tail of ChunkedEllpack's slice container, which TNL
  leaves uninitialised, excepted), in every layout and both value types;
* TNL loads the files written here exactly as it loads its own, and the
  files TNL writes load here into TNL's arrays — including a matrix whose
  rows were given more capacity than they use (TNL's own ChunkedEllpack load
  swaps two mapping arrays that its save writes in another order; they are
  read here as written);
* broken files are refused (wrong magic, truncation, another matrix type,
  inconsistent arrays).
"""
import struct

import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

LAYOUTS = {"csr": "CSR", "ellpack": "Ellpack", "slicedellpack": "SlicedEllpack", "chunkedellpack": "ChunkedEllpack",
           "biellpack": "BiEllpack", "slicedellpack16": "SlicedEllpack"}
REAL = {"f64": "double", "f32": "float"}


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference()


def _mask_chunked_tail(data: bytes, rows: int) -> bytes:
    """Zero the slice entries past numberOfSlices (TNL leaves them uninitialised)."""
    tag = b"ChunkedEllpackSliceInfo<int>, [any_device], int, [any_allocator] >"
    p = data.index(tag) + len(tag)
    n = struct.unpack_from("<i", data, p)[0]
    nsl = struct.unpack_from("<i", data, p + 4 + 16 * n)[0]
    body = bytearray(data)
    for k in range(nsl, n):
        body[p + 4 + 16 * k:p + 4 + 16 * (k + 1)] = bytes(16)
    return bytes(body)


def _arrays(M, want):
    return {k: M.export(k) for k in want}


def _same(got, want, fmt):
    for k in want:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        if k == "values":
            g = g.astype(np.float64)
        assert g.shape == w.shape and np.array_equal(g, w), (fmt, k)


@pytest.mark.parametrize("name", ["poisson_7x5", "irregular_zeros_empty", "irregular_long"])
@pytest.mark.parametrize("fmt", sorted(LAYOUTS))
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_save_matches_tnl_and_loads_both_ways(b2s_lib, cuda, ref, tmp_path, name, fmt, real):
    csr = F.csr(name)
    n = len(csr[0]) - 1
    ss = F.SLICE.get(fmt, 0)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=LAYOUTS[fmt], real=REAL[real], slice_size=ss)
    ours, theirs = tmp_path / "ours.tnl", tmp_path / "tnl.tnl"
    M.save(ours)
    ref.save(fmt, "col", csr, theirs, real)
    a, b = ours.read_bytes(), theirs.read_bytes()
    if fmt == "chunkedellpack":
        a, b = _mask_chunked_tail(a, n), _mask_chunked_tail(b, n)
    assert a == b
    want = ref.convert(fmt, "col", csr, real)
    # TNL reads our file exactly as it reads its own, and gets its arrays back
    # (ChunkedEllpack excepted: TNL's load takes the mapping arrays in another
    # order than its save writes them, ChunkedEllpack.hpp:379-407)
    got, own = ref.load(fmt, "col", ours, real), ref.load(fmt, "col", theirs, real)
    assert got is not None and own is not None
    for k in want:
        assert np.array_equal(got[k], own[k]), (fmt, k)
        if fmt != "chunkedellpack":
            assert np.array_equal(got[k], want[k]), (fmt, k)
    # we read TNL's file
    L = b2s_lib.SparseMatrix.load(theirs, slice_size=ss)
    _same(_arrays(L, want), want, fmt)
    x = np.random.default_rng(1).uniform(-1, 1, csr[3]).astype(np.float64 if real == "f64" else np.float32)
    y1, y2 = np.zeros(n, x.dtype), np.zeros(n, x.dtype)
    M.vectorProduct(x, y1)
    L.vectorProduct(x, y2)
    assert np.array_equal(y1, y2)


@pytest.mark.parametrize("fmt", sorted(LAYOUTS))
def test_load_rows_with_spare_capacity(b2s_lib, cuda, ref, oracle, tmp_path, fmt):
    """setRowCapacities larger than the rows' elements (TNL keeps the spare
    slots as padding): the file's layout is taken as stored."""
    g = np.random.default_rng(3)
    rows, cols, n = 120, 90, 700
    ri, ci = g.integers(0, rows, n), g.integers(0, cols, n)
    v = g.normal(size=n)
    caps = np.bincount(ri, minlength=rows) + g.integers(0, 4, rows)
    path = tmp_path / "caps.tnl"
    want = ref.from_coo(fmt, "col", rows, cols, ri, ci, v, caps=caps, save_to=path)
    L = b2s_lib.SparseMatrix.load(path, slice_size=F.SLICE.get(fmt, 0))
    if fmt == "csr":  # TNL's CSR keeps the spare slots (column -1); the rows here hold the elements
        keep = want["columnIndexes"] != -1
        assert np.array_equal(L.export("columnIndexes"), want["columnIndexes"][keep])
        assert np.array_equal(L.export("values"), want["values"][keep])
    else:
        _same(_arrays(L, want), want, fmt)


def test_broken_files_are_refused(b2s_lib, cuda, ref, tmp_path):
    csr = F.csr("poisson_7x5")
    good = tmp_path / "good.tnl"
    ref.save("slicedellpack", "col", csr, good)
    data = good.read_bytes()
    cases = {
        "magic": b"XNLMN" + data[5:],
        "truncated": data[: len(data) // 2],
        "empty": b"",
        "other_type": data.replace(b"SlicedEllpack<", b"SlicedEllpock<"),
    }
    for name, blob in cases.items():
        p = tmp_path / f"{name}.tnl"
        p.write_bytes(blob)
        with pytest.raises(b2s_lib.B2SError) as e:
            b2s_lib.SparseMatrix.load(p)
        assert e.value.status in (b2s_lib.INVALID_ARG, b2s_lib.IO_ERROR), name
    # a slice offset pointing past the storage
    tag = b"Containers::Array< int, [any_device], int, [any_allocator] >"
    p2 = data.rindex(tag)  # sliceSegmentSizes; the slice offsets are the array before it
    p1 = data.rindex(tag, 0, p2)
    off = p1 + len(tag) + 4
    blob = bytearray(data)
    struct.pack_into("<i", blob, off + 4, 10 ** 8)
    p = tmp_path / "offsets.tnl"
    p.write_bytes(bytes(blob))
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.load(p)
    assert e.value.status == b2s_lib.INVALID_ARG
    # a BiEllpack row permutation that sends two rows of a strip to one place
    bi = tmp_path / "bi.tnl"
    ref.save("biellpack", "col", csr, bi)
    data = bi.read_bytes()
    p2 = data.rindex(tag)  # groupPointers; rowPermArray is the array before it
    p1 = data.rindex(tag, 0, p2)
    off = p1 + len(tag) + 4
    blob = bytearray(data)
    struct.pack_into("<i", blob, off + 4, struct.unpack_from("<i", blob, off)[0])
    p = tmp_path / "perm.tnl"
    p.write_bytes(bytes(blob))
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.load(p)
    assert e.value.status == b2s_lib.INVALID_ARG and "permutation" in str(e.value)
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.load(tmp_path / "absent.tnl")
    assert e.value.status == b2s_lib.IO_ERROR
