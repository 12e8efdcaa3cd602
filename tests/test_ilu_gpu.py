"""ILU(0) on the device (B2S_PRECOND_ILU0) against TNL's own
Preconditioners::ILU0 (Devices::Host, compiled from the reference headers).

* one application M^-1 b equals TNL's update + solve bit for bit, FP64 and
  FP32, host and device vectors, in place, and on padded layouts (the same
  rows in storage order);
* repeated applications (new epochs) give the same bits;
* a missing diagonal entry or unsorted columns are refused as TNL's CUDA path
  refuses them ("A(i, i) is missing");
* CG, BiCGStab and GMRES preconditioned by ILU(0) match TNL's runs with ILU0:
  converged flag, iterations within max(2, 2 %), solution within 1e-8 at
  convergence residue 1e-10.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REAL = {"f64": ("double", np.float64), "f32": ("float", np.float32)}


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    return Reference()


def _cases():
    from b2s import workloads as W
    g = np.random.default_rng(8)
    n = 3000  # random sparse, diagonally dominant, nonsymmetric pattern
    lens = g.integers(1, 12, n)
    rows = [np.unique(np.concatenate([[i], g.choice(n, L, replace=False)])) for i, L in enumerate(lens)]
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    col = np.concatenate(rows).astype(np.int32)
    val = g.uniform(-1, 1, len(col))
    val[col == np.repeat(np.arange(n), np.diff(off))] = 20.0
    return {"convdiff": W.convdiff3d(16, seed=4), "diffusion": W.diffusion3d(18, seed=3),
            "poisson2d": W.poisson2d(60), "random": (off, col, val, n)}


@pytest.mark.parametrize("name", ["convdiff", "diffusion", "poisson2d", "random"])
@pytest.mark.parametrize("real", ["f64", "f32"])
def test_ilu0_apply_bitwise_vs_tnl(b2s_lib, cuda, ref, name, real):
    csr = _cases()[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(1).uniform(-1, 1, n)
    want = ref.ilu0_apply(csr, b, real)
    rname, dt = REAL[real]
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], real=rname)
    P = b2s_lib.Preconditioner(M, "ilu0")
    x = np.zeros(n, dt)
    P.solve(b.astype(dt), x)
    assert np.array_equal(x.astype(np.float64), want), np.max(np.abs(x - want))
    tdt = cuda.float64 if real == "f64" else cuda.float32
    bd = cuda.tensor(b, dtype=tdt, device="cuda")
    for _ in range(3):  # new epochs, same bits; in place
        xd = bd.clone()
        P.solve(xd, xd)
        assert np.array_equal(xd.cpu().numpy().astype(np.float64), want)


@pytest.mark.parametrize("fmt", ["Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"])
def test_ilu0_on_padded_layouts(b2s_lib, cuda, ref, fmt):
    csr = _cases()["convdiff"]
    n = len(csr[0]) - 1
    b = np.random.default_rng(2).uniform(-1, 1, n)
    want = ref.ilu0_apply(csr, b)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=fmt)
    x = np.zeros(n)
    b2s_lib.Preconditioner(M, "ilu0").solve(b, x)
    assert np.array_equal(x, want)


def test_ilu0_refuses_missing_diagonal_and_unsorted_rows(b2s_lib, cuda):
    off = np.array([0, 2, 3, 5], np.int32)
    col = np.array([0, 2, 0, 1, 2], np.int32)  # row 1 has no (1, 1)
    M = b2s_lib.SparseMatrix.from_csr(off, col, np.ones(5), 3)
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.Preconditioner(M, "ilu0")
    assert e.value.status == b2s_lib.INVALID_ARG and "A(1, 1) is missing" in str(e.value)
    col = np.array([2, 0, 1, 2, 1], np.int32)  # row 0 unsorted
    M = b2s_lib.SparseMatrix.from_csr(off, col, np.ones(5), 3)
    with pytest.raises(b2s_lib.B2SError) as e:
        b2s_lib.Preconditioner(M, "ilu0")
    assert e.value.status == b2s_lib.INVALID_ARG


@pytest.mark.parametrize("solver,name", [("cg", "diffusion"), ("cg", "poisson2d"), ("bicgstab", "convdiff"),
                                         ("gmres", "convdiff"), ("bicgstab", "random"), ("gmres", "random")])
def test_solvers_with_ilu0_vs_tnl(b2s_lib, cuda, ref, solver, name):
    csr = _cases()[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    want = ref.solve(solver, csr, b, rtol=1e-10, precond=2, gmres_variant="MGSR", restart_min=30, restart_max=30)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = {"cg": b2s_lib.CG, "bicgstab": b2s_lib.BICGStab, "gmres": b2s_lib.GMRES}[solver]()
    s.setMatrix(M)
    s.setPreconditioner("ilu0")
    s.setConvergenceResidue(1e-10)
    s.setup({"gmres-variant": "MGSR", "gmres-restarting-min": 30, "gmres-restarting-max": 30})
    for _ in range(2):  # the second solve replays the captured iterations
        x = cuda.zeros(n, dtype=cuda.float64, device="cuda")
        ok = s.solve(cuda.tensor(b, device="cuda"), x)
        assert ok == want["converged"]
        assert abs(s.getIterations() - want["iterations"]) <= max(2, 0.02 * want["iterations"])
        xh = x.cpu().numpy()
        assert np.max(np.abs(xh - want["x"])) / np.max(np.abs(want["x"])) <= 1e-8


def test_ilu0_cuts_iterations(b2s_lib, cuda):
    """ILU(0) against Jacobi on the variable-coefficient diffusion matrix."""
    from b2s import workloads as W
    csr = W.diffusion3d(24, seed=3)
    n = len(csr[0]) - 1
    b = cuda.tensor(W.uniform(n, 5), device="cuda")
    its = {}
    for pre in ("diagonal", "ilu0"):
        M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
        s = b2s_lib.CG()
        s.setMatrix(M)
        s.setPreconditioner(pre)
        s.setConvergenceResidue(1e-10)
        x = cuda.zeros(n, dtype=cuda.float64, device="cuda")
        assert s.solve(b, x)
        its[pre] = s.getIterations()
    assert its["ilu0"] < 0.75 * its["diagonal"], its
