"""MatrixMarket input (MatrixReader::readMtx semantics) and the assembly
restatement of the oracle, on the CPU.

* the oracle's setElement / addElement assembly (b2so_from_coo) equals TNL's
  own (setRowCapacities + setElement / addElement through the compiled
  reference) array for array, in every layout and both value types;
* b2s_mtx_read (the library's host parser) followed by that assembly equals
  TNL's MatrixReader::readMtx array for array — comments, blank lines,
  leading spaces, duplicates, explicit zeros, symmetric files;
* every file TNL's reader rejects is rejected, with TNL's message where TNL
  gives one.
"""
import numpy as np
import pytest

LAYOUTS = ["csr", "ellpack", "slicedellpack", "chunkedellpack", "biellpack", "slicedellpack16"]


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    try:
        return Reference()
    except FileNotFoundError:
        pytest.skip("oracle/_ref (TNL compiled from the reference headers) is not built")


def _write(path, text):
    path.write_bytes(text.encode())
    return path


def _random_mtx(rows, cols, n, seed, symmetric=False, dups=True, zeros=True):
    g = np.random.default_rng(seed)
    r = g.integers(1, rows + 1, n)
    c = g.integers(1, cols + 1, n)
    if symmetric:
        r, c = np.maximum(r, c), np.minimum(r, c)
    if not dups:
        key = np.unique(r.astype(np.int64) * (cols + 1) + c)
        r, c = key // (cols + 1), key % (cols + 1)
        g.shuffle(idx := np.arange(len(r)))
        r, c = r[idx], c[idx]
    v = g.normal(size=len(r))
    if zeros:
        v[::13] = 0.0
    kind = "symmetric" if symmetric else "general"
    lines = [f"%%MatrixMarket matrix coordinate real {kind}", "% a comment", f"{rows} {cols} {len(r)}"]
    for i, (a, b, x) in enumerate(zip(r, c, v)):
        sep = "   " if i % 7 == 0 else " "
        lines.append(f"{'  ' if i % 5 == 0 else ''}{a}{sep}{b} {float(x)!r}")
        if i % 11 == 0:
            lines.append("")        # blank lines between elements are skipped
        if i % 17 == 0:
            lines.append("%% comment inside the element list")
    return "\n".join(lines) + "\n"


def test_oracle_assembly_matches_tnl(oracle, ref):
    g = np.random.default_rng(7)
    rows, cols, n = 70, 45, 900
    ri, ci = g.integers(0, rows, n), g.integers(0, cols, n)
    v = g.normal(size=n)
    v[::9] = 0.0
    for fmt in LAYOUTS + ["slicedellpack8", "slicedellpack64"]:
        for org in ("col", "row"):
            for real in ("f64", "f32"):
                for add in (False, True):
                    a = oracle.from_coo(fmt, org, rows, cols, ri, ci, v, add, real)
                    b = ref.from_coo(fmt, org, rows, cols, ri, ci, v, add, real)
                    assert a.keys() == b.keys()
                    for k in a:
                        assert np.array_equal(a[k], b[k]), (fmt, org, real, add, k)


@pytest.mark.parametrize("case", ["general", "symmetric", "no_dups", "square_dense_row"])
def test_mtx_read_matches_tnl_reader(b2s_lib, oracle, ref, tmp_path, case):
    if case == "general":
        text = _random_mtx(60, 50, 700, 1)
    elif case == "symmetric":
        text = _random_mtx(80, 80, 500, 2, symmetric=True)
    elif case == "no_dups":
        text = _random_mtx(40, 90, 600, 3, dups=False, zeros=False)
    else:  # one row with every column, no trailing newline
        text = "%%MatrixMarket matrix coordinate real general\n3 6 8\n" + "".join(
            f"2 {c} {c * 0.5}\n" for c in range(6, 0, -1)) + "1 1 1.0\n3 3 -2e-300"
    p = _write(tmp_path / "m.mtx", text)
    m = b2s_lib.mtx_read(p)
    assert m["symmetric"] == (case == "symmetric")
    for fmt in LAYOUTS:
        for real in ("f64", "f32"):
            want = ref.read_mtx(fmt, "col", p, real)
            assert want is not None
            got = oracle.from_coo(fmt, "col", m["rows"], m["cols"], m["row_indexes"], m["column_indexes"],
                                  m["values"], False, real)
            assert got.keys() == want.keys()
            for k in got:
                assert np.array_equal(got[k], want[k]), (case, fmt, real, k)


BAD = {
    "empty": "",
    "no_banner": "%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1\n",
    "array": "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "complex": "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",
    "pattern": "%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n",
    "hermitian": "%%MatrixMarket matrix coordinate real hermitian\n2 2 1\n1 1 1\n",
    "not_matrix": "%%MatrixMarket vector coordinate real general\n2 2 1\n1 1 1\n",
    "short_banner": "%%MatrixMarket matrix coordinate real\n2 2 1\n1 1 1\n",
    "crlf_banner": "%%MatrixMarket matrix coordinate real general\r\n2 2 1\r\n1 1 1\r\n",
    "dims_two_tokens": "%%MatrixMarket matrix coordinate real general\n2 2\n1 1 1\n",
    "dims_zero": "%%MatrixMarket matrix coordinate real general\n0 2 0\n",
    "blank_before_dims": "%%MatrixMarket matrix coordinate real general\n\n2 2 1\n1 1 1\n",
    "no_dims": "%%MatrixMarket matrix coordinate real general\n% only comments\n",
    "element_two_tokens": "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n2 2\n",
    "element_four_tokens": "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1 7\n",
    "tabs": "%%MatrixMarket matrix coordinate real general\n2 2 1\n1\t1\t1\n",
    "row_out_of_range": "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",
    "col_out_of_range": "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 3 1\n",
    "row_over_capacity": "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n1 2 1\n1 1 5\n",
}


@pytest.mark.parametrize("name", sorted(BAD))
def test_mtx_read_rejects_what_tnl_rejects(b2s_lib, ref, tmp_path, name):
    p = _write(tmp_path / f"{name}.mtx", BAD[name])
    assert ref.read_mtx("csr", "col", p) is None  # TNL's reader throws
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.mtx_read(p)
    assert e.value.status in (b2s_lib.INVALID_ARG, b2s_lib.IO_ERROR)


def test_mtx_read_rejects_indexes_below_one(b2s_lib, tmp_path):
    """TNL's reader does not check for row or column 0 (it then writes before
    its row-length array); these files are rejected here."""
    for text in ("%%MatrixMarket matrix coordinate real general\n2 2 1\n0 1 1\n",
                 "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 -1 1\n"):
        p = _write(tmp_path / "z.mtx", text)
        with pytest.raises(b2s_lib.B2SError) as e:
            b2s_lib.mtx_read(p)
        assert e.value.status == b2s_lib.INVALID_ARG


def test_mtx_read_missing_file(b2s_lib, tmp_path):
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.mtx_read(tmp_path / "absent.mtx")
    assert e.value.status == b2s_lib.IO_ERROR


def test_mtx_read_parallel_chunks_keep_file_order(b2s_lib, tmp_path):
    """A file above the single-thread threshold is parsed in line-aligned
    chunks; the triplets come back in file order."""
    g = np.random.default_rng(5)
    n = 120000
    r, c = g.integers(1, 5001, n), g.integers(1, 4001, n)
    v = g.normal(size=n)
    body = "".join(f"{a} {b} {float(x)!r}\n" for a, b, x in zip(r, c, v))
    p = _write(tmp_path / "big.mtx", f"%%MatrixMarket matrix coordinate real general\n5000 4000 {n}\n" + body)
    m = b2s_lib.mtx_read(p)
    assert np.array_equal(m["row_indexes"], r - 1)
    assert np.array_equal(m["column_indexes"], c - 1)
    assert np.array_equal(m["values"], v)
