"""Preconditioners::ILUT on the device against TNL's own ILUT (Devices::Host,
compiled from the reference headers; ILUT.hpp:33-289), through the C ABI.

TNL provides ILUT on the host only (its Devices::Cuda specialization throws);
the library runs TNL's factorization on the host and applies the factors on
the device. The reference's factorization has choices of its own that the
tests pin through its results: w_k is divided by A_kk and U's row k is
subtracted with its diagonal, and at most ceil(size / 2) heap candidates are
kept per factor row. Criteria:

* M^-1 b bit for bit equal to TNL's ILUT::solve, FP64 and FP32, for
  p in {0, 1, 2, 5} and thresholds 0 to 0.05, on a nonsymmetric and a
  symmetric matrix (equal magnitudes: ties in the heaps), in CSR and padded
  layouts, and for a SymmetricMatrix;
* GMRES with ILUT converges as TNL's host GMRES does (one OpenMP thread), in
  as many iterations (max(2, 2 %)), to a true residual within 10x of TNL's
  and a solution within 1e-5 of TNL's; BiCGStab with ILUT converges as
  TNL's does, to a true residual within 10x of TNL's. (The reference's ILUT
  is a weak preconditioner: a preconditioned residue of 1e-10 leaves ~1e-7
  in x, and BiCGStab's iteration count with it moves with the rounding of the
  reductions — TNL's own count changes with its thread count.)
* mixed precision with ILUT and a negative p are refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PARAMS = [(0, 1e-4), (1, 0.05), (2, 1e-3), (5, 0.0)]


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference()


def _matrices():
    from b2s import workloads as W
    g = np.random.default_rng(11)
    cd = W.convdiff3d(6, seed=7)
    off, col, val, nc = cd
    cd = (off, col, val * g.uniform(0.8, 1.2, len(val)), nc)
    return {"convdiff": cd, "poisson": W.poisson2d(18)}


def _tnl_apply(ref, csr, p, tau, b, real):
    h, _ = ref.ilut(csr, p=p, tau=tau, real=real)
    try:
        return ref.ilut_solve(h, b)
    finally:
        ref.ilut_destroy(h)


@pytest.mark.parametrize("name", ["convdiff", "poisson"])
@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("p,tau", PARAMS)
def test_application_bitwise_vs_tnl(b2s_lib, cuda, ref, name, real, p, tau):
    csr = _matrices()[name]
    if real == "f32":
        csr = (csr[0], csr[1], csr[2].astype(np.float32).astype(np.float64), csr[3])
    n = len(csr[0]) - 1
    dt = np.float64 if real == "f64" else np.float32
    rname = "double" if real == "f64" else "float"
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], real=rname)
    P = b2s_lib.Preconditioner(M, "ilut", p=p, threshold=tau)
    g = np.random.default_rng(3)
    for _ in range(2):
        b = g.uniform(-1, 1, n).astype(dt)
        want = _tnl_apply(ref, csr, p, tau, b.astype(np.float64), real).astype(dt)
        x = np.zeros(n, dt)
        P.solve(b, x)  # host vectors
        assert np.array_equal(x, want), np.max(np.abs(x - want))
        xd = cuda.zeros(n, dtype=cuda.float64 if real == "f64" else cuda.float32, device="cuda")
        P.solve(cuda.tensor(b, device="cuda"), xd)  # device vectors
        assert np.array_equal(xd.cpu().numpy(), want)


@pytest.mark.parametrize("layout", ["Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"])
def test_padded_layouts_and_symmetric(b2s_lib, cuda, ref, layout):
    csr = _matrices()["poisson"]
    off, col, val, n = csr
    b = np.random.default_rng(4).uniform(-1, 1, n)
    want = _tnl_apply(ref, csr, 2, 1e-3, b, "f64")
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, n, segments=layout)
    x = np.zeros(n)
    b2s_lib.Preconditioner(M, "ilut", p=2, threshold=1e-3).solve(b, x)
    assert np.array_equal(x, want)
    rows = np.repeat(np.arange(n), np.diff(off))
    keep = col <= rows
    loff = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.int32)
    S = b2s_lib.SparseMatrix.from_csr(loff, col[keep], val[keep], n, segments=layout, symmetric=True)
    x = np.zeros(n)
    b2s_lib.Preconditioner(S, "ilut", p=2, threshold=1e-3).solve(b, x)
    assert np.array_equal(x, want)


@pytest.mark.parametrize("solver,tnl", [("BICGStab", "bicgstab"), ("GMRES", "gmres")])
@pytest.mark.parametrize("p,tau", [(0, 1e-4), (3, 1e-3)])
def test_solvers_with_ilut_vs_tnl(b2s_lib, cuda, ref, solver, tnl, p, tau):
    csr = _matrices()["convdiff"]
    n = len(csr[0]) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    ref.lib.tnlref_set_ilut(p, tau)
    threads = ref.threads()
    ref.set_threads(1)
    try:
        want = ref.solve(tnl, csr, b, rtol=1e-10, precond=3, gmres_variant="MGSR", restart_min=30, restart_max=30)
    finally:
        ref.lib.tnlref_set_ilut(0, 1e-4)
        ref.set_threads(threads)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = getattr(b2s_lib, solver)()
    s.setMatrix(M)
    s.setPreconditioner("ilut")
    s.setConvergenceResidue(1e-10)
    assert s.setup({"ilut-p": p, "ilut-threshold": tau, "gmres-restarting-min": 30, "gmres-restarting-max": 30})
    x = np.zeros(n)
    ok = s.solve(b, x)
    assert ok == want["converged"] and ok
    if solver == "GMRES":
        assert abs(s.getIterations() - want["iterations"]) <= max(2, 0.02 * want["iterations"])
        assert np.max(np.abs(x - want["x"])) / np.max(np.abs(want["x"])) <= 1e-5

    def true_res(v):
        off, col, val, _ = csr
        ax = np.add.reduceat(val * v[col], off[:-1]) if len(val) else np.zeros(n)
        return np.linalg.norm(b - ax) / np.linalg.norm(b)
    assert true_res(x) <= 10 * true_res(want["x"]) + 1e-13


def test_refusals(b2s_lib, cuda):
    csr = _matrices()["poisson"]
    n = len(csr[0]) - 1
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.Preconditioner(M, "ilut", p=-1)
    assert e.value.status == b2s_lib.INVALID_ARG
    s = b2s_lib.CG()
    s.setMatrix(M)
    s.setPreconditioner("ilut")
    s.setPrecision(True)
    with pytest.raises(b2s_lib.B2SError) as e:
        s.solve(np.ones(n), np.zeros(n))
    assert e.value.status == b2s_lib.UNSUPPORTED
