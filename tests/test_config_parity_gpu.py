"""Parity with TNL at the full sizes of the benchmarked workloads.

The small fixtures of the other test files pin every layout and solver
against TNL on matrices of up to a few hundred rows; here the same properties
are checked on the matrices the benchmark times:

* SpMV sweep matrices (3D 7-point Laplacian 128^3, 2.1M rows; seeded
  irregular log-normal matrix, 2M rows): every layout's storage arrays equal
  TNL's own arrays bit for bit (SHA-256 digests of TNL's arrays, committed by
  tests/golden/make_config_layouts.py), Ellpack of the irregular matrix is
  refused as TNL refuses it (more than 2^31 slots), and every layout's FP64
  product is within 1e-12 relative (max |y - y_ref| / max |y_ref|) of TNL's
  Devices::Host CSR product computed here, FP32 within 1e-5 of TNL's FP32
  product;
* the 128^3 Laplacian as a Multidiagonal matrix: its values array equals TNL's
  own MultidiagonalMatrix (ColumnMajor, built here by TNL's setElement with the
  same diagonals) bit for bit, and its FP64 / FP32 product is within 1e-12 /
  1e-5 of TNL's Multidiagonal product; the irregular matrix (millions of
  diagonals) is refused;
* CG on the 256^2 Poisson system (b = A*1, rtol 1e-8): iteration count within
  max(2, 2 %) of TNL's host CG and x within 1e-8 relative of TNL's x;
* the mixed-precision cases (CG on 160^3 variable-coefficient diffusion,
  BiCGStab and GMRES(30) on 128^3 upwind convection-diffusion, rtol 1e-10):
  FP64 and mixed solutions within 1e-7 relative of TNL's host FP64 solution
  by the same method, true FP64 residual <= 1e-10, FP64 iteration counts
  within 2 % of TNL's;
* the batched workload (4,096 shifted 2D Laplacians, Jacobi-PCG to rtol 1e-8):
  a sample of systems from the smallest to the largest against TNL's host CG
  with the Diagonal preconditioner, iterations within max(2, 2 %) and x within
  1e-7 relative.

TNL's host code runs from oracle/_ref (built from the reference headers).
"""
import hashlib
import json
import os
from functools import lru_cache

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

SEGMENTS = {"csr": "CSR", "ellpack": "Ellpack", "slicedellpack": "SlicedEllpack",
            "chunkedellpack": "ChunkedEllpack", "biellpack": "BiEllpack"}
CHUNK = 1 << 24


@lru_cache(None)
def digests():
    return json.loads((GOLDEN / "config_layouts.json").read_text())


@lru_cache(None)
def reference():
    from oracle import Reference
    R = Reference()
    R.set_threads(len(os.sched_getaffinity(0)))
    return R


@lru_cache(2)
def matrix(name):
    from b2s import workloads as W
    csr = W.laplace3d(128) if name == "laplace3d_128" else W.irregular(2_000_000, seed=2)
    want = digests()[name]["csr_sha256"]
    got = {"offsets": hashlib.sha256(np.ascontiguousarray(csr[0], np.int32).tobytes()).hexdigest(),
           "columns": hashlib.sha256(np.ascontiguousarray(csr[1], np.int32).tobytes()).hexdigest(),
           "values": hashlib.sha256(np.ascontiguousarray(csr[2], np.float64).tobytes()).hexdigest()}
    assert got == want, "the seeded generator does not reproduce the matrix the digests were made from"
    return csr


def _rel(got, want):
    return float(np.max(np.abs(got - want)) / max(float(np.max(np.abs(want))), 1e-300))


def _digest(M, name, length):
    d = hashlib.sha256()
    for first in range(0, length, CHUNK):
        d.update(M.export_range(name, first, min(CHUNK, length - first)).tobytes())
    return d.hexdigest()


@pytest.mark.parametrize("name", ["laplace3d_128", "irregular_2m"])
@pytest.mark.parametrize("fmt", list(SEGMENTS))
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_full_size_layout_matches_tnl(b2s_lib, cuda, name, fmt, real):
    want = digests()[name][f"{fmt}/{real}"]
    csr = matrix(name)
    mk = lambda: b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=SEGMENTS[fmt],
                                               real="double" if real == "f64" else "float")
    if want.get("refused"):
        with pytest.raises(b2s_lib.B2SError) as e:
            mk()
        assert e.value.status == b2s_lib.INDEX_OVERFLOW
        return
    M = mk()
    assert M.getStorageSize() == want["storage"]
    length = want["digest_length"]
    if fmt == "biellpack":  # slots past the addressed part are padding, as in TNL (checked by the generator)
        tail = M.export_range("columnIndexes", length, min(CHUNK, want["storage"] - length))
        assert np.all(tail == -1)
    assert _digest(M, "columnIndexes", length) == want["columnIndexes"]
    assert _digest(M, "values", length) == want["values"]
    for k, m in want["meta"].items():
        a = M.export(k).astype(np.int64)
        assert len(a) == m["len"] and hashlib.sha256(a.tobytes()).hexdigest() == m["sha256"], k
    del M
    cuda.cuda.empty_cache()


@lru_cache(4)
def tnl_product(name, real):
    from b2s import workloads as W
    csr = matrix(name)
    x = W.uniform(csr[3], 1)
    if real == "f32":
        x = x.astype(np.float32).astype(np.float64)
    return x, reference().spmv("csr", "col", csr, x, real=real)


@pytest.mark.parametrize("name", ["laplace3d_128", "irregular_2m"])
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_full_size_spmv_vs_tnl_host(b2s_lib, cuda, name, real):
    csr = matrix(name)
    x, want = tnl_product(name, real)
    dt = cuda.float64 if real == "f64" else cuda.float32
    tol = 1e-12 if real == "f64" else 1e-5
    xd = cuda.tensor(x, dtype=dt, device="cuda")
    yd = cuda.empty(len(want), dtype=dt, device="cuda")
    r = "double" if real == "f64" else "float"
    variants = [(seg, {}) for seg in SEGMENTS.values()]
    variants += [("CSR", {"csr_row_groups": False}), ("CSR", {"csr_kernel": "CSRScalar"}),
                 ("CSR", {"csr_kernel": "CSRVector", "threads_per_row": 8})]
    checked = 0
    for seg, kw in variants:
        try:
            M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=seg, real=r, **kw)
        except b2s_lib.B2SError as e:
            assert seg == "Ellpack" and name == "irregular_2m" and e.status == b2s_lib.INDEX_OVERFLOW
            continue
        yd.fill_(np.nan)
        M.vectorProduct(xd, yd)
        err = _rel(yd.cpu().numpy().astype(np.float64), want)
        assert err <= tol, (seg, kw, err)
        checked += 1
        del M
        cuda.cuda.empty_cache()
    assert checked >= 7


@pytest.mark.parametrize("real", ["f64", "f32"])
def test_full_size_multidiagonal_vs_tnl(b2s_lib, cuda, real):
    from b2s import workloads as W
    csr = matrix("laplace3d_128")
    off, col, val, n = csr
    r = "double" if real == "f64" else "float"
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, n, segments="Multidiagonal", real=r)
    offsets = M.export("diagonalsOffsets")
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    d = np.searchsorted(offsets, col.astype(np.int64) - rows)
    dense = np.zeros((n, len(offsets)))
    dense[rows, d] = val
    R = reference()
    h = R.multidiagonal(n, n, offsets, dense, real=real)
    try:
        assert np.array_equal(M.export("values").astype(np.float64), R.mdiag_values(h))
        x = W.uniform(n, 1)
        if real == "f32":
            x = x.astype(np.float32).astype(np.float64)
        want = R.mdiag_spmv(h, x, np.zeros(n))
    finally:
        R.mdiag_destroy(h)
    dt = cuda.float64 if real == "f64" else cuda.float32
    yd = cuda.full((n,), float("nan"), dtype=dt, device="cuda")
    M.vectorProduct(cuda.tensor(x, dtype=dt, device="cuda"), yd)
    assert _rel(yd.cpu().numpy().astype(np.float64), want) <= (1e-12 if real == "f64" else 1e-5)
    del M
    irr = matrix("irregular_2m")
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.SparseMatrix.from_csr(*irr[:3], irr[3], segments="Multidiagonal", real=r)
    assert e.value.status == b2s_lib.UNSUPPORTED
    cuda.cuda.empty_cache()


def test_poisson256_cg_vs_tnl_host(b2s_lib, cuda):
    from b2s import workloads as W
    R = reference()
    csr = W.poisson2d(256)
    n = len(csr[0]) - 1
    b = R.spmv("csr", "col", csr, np.ones(n))
    t = R.solve("cg", csr, b, rtol=1e-8)
    A = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = b2s_lib.CG()
    s.setMatrix(A)
    s.setConvergenceResidue(1e-8)
    x = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    assert s.solve(cuda.tensor(b, device="cuda"), x)
    its = s.getIterations()
    assert t["converged"] and abs(its - t["iterations"]) <= max(2, 0.02 * t["iterations"]), (its, t["iterations"])
    assert _rel(x.cpu().numpy(), t["x"]) <= 1e-8


CASES = [("diffusion3d_160", "cg"), ("convdiff3d_128", "bicgstab"), ("convdiff3d_128", "gmres")]


@lru_cache(2)
def system(mname):
    from b2s import workloads as W
    csr = W.diffusion3d(160, seed=3) if mname.startswith("diffusion") else W.convdiff3d(128, seed=4)
    return csr, W.uniform(len(csr[0]) - 1, 11)


@lru_cache(4)
def tnl_solution(mname, kind):
    csr, b = system(mname)
    t = reference().solve(kind, csr, b, rtol=1e-10, gmres_variant="CGSR", restart_min=30, restart_max=30)
    assert t["converged"]
    return t


@pytest.mark.parametrize("mname,kind", CASES)
def test_full_size_solves_vs_tnl_host(b2s_lib, cuda, mname, kind):
    csr, bh = system(mname)
    t = tnl_solution(mname, kind)
    A = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], keep_fp32_copy=True)
    b = cuda.tensor(bh, device="cuda")
    for mixed in (False, True):
        s = {"cg": b2s_lib.CG, "bicgstab": b2s_lib.BICGStab, "gmres": b2s_lib.GMRES}[kind]()
        s.setMatrix(A)
        s.setConvergenceResidue(1e-10)
        s.setup({"gmres-variant": "CGSR", "gmres-restarting-min": 30, "gmres-restarting-max": 30})
        s.setPrecision(mixed)
        x = cuda.zeros(A.getRows(), dtype=cuda.float64, device="cuda")
        assert s.solve(b, x), (kind, mixed)
        err = _rel(x.cpu().numpy(), t["x"])
        assert err <= 1e-7, (kind, mixed, err)
        assert s.report.true_residual <= 1e-10, (kind, mixed, s.report.true_residual)
        if not mixed:
            its = s.getIterations()
            assert abs(its - t["iterations"]) <= max(2, 0.02 * t["iterations"]), (kind, its, t["iterations"])
    del A
    cuda.cuda.empty_cache()


def test_batched_workload_sample_vs_tnl_host(b2s_lib, cuda):
    from b2s import workloads as W
    off, col, val, rp, nr = W.batched_poisson2d(4096, seed=5)
    bt = b2s_lib.BatchedCG(cuda.from_numpy(off).cuda(), cuda.from_numpy(col).cuda(), cuda.from_numpy(val).cuda(),
                           rp, nr, tol=1e-8)
    B = cuda.tensor(np.random.default_rng(9).uniform(-1, 1, bt.vector_length), device="cuda")
    X = cuda.zeros_like(B)
    assert bt.solve(B, X)
    its, _, sts = bt.results()
    Bh, Xh = B.cpu().numpy(), X.cpu().numpy()
    R = reference()
    order = np.argsort(np.diff(rp), kind="stable")
    for i in np.linspace(0, len(order) - 1, 6).astype(int):
        s = int(order[i])
        csr = W.batch_system(off, col, val, rp, s)
        n, k = csr[3], int(nr[s])
        blk = slice(int(bt.vec_off[s]), int(bt.vec_off[s + 1]))
        for j in range(k):
            t = R.solve("cg", csr, np.ascontiguousarray(Bh[blk].reshape(n, k)[:, j]), rtol=1e-8, precond=True)
            slot = int(bt.rhs_off[s]) + j
            assert t["converged"] and sts[slot] == b2s_lib.OK
            assert abs(int(its[slot]) - t["iterations"]) <= max(2, 0.02 * t["iterations"]), (s, j, its[slot],
                                                                                              t["iterations"])
            err = _rel(Xh[blk].reshape(n, k)[:, j], t["x"])
            assert err <= 1e-7, (s, j, err)
