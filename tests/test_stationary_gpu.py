"""Solvers::Linear::Jacobi and SOR on the device against TNL's own solvers
(Devices::Host, compiled from the reference headers; Jacobi.hpp:67-128,
SOR.hpp:66-118), through the C ABI.

* SOR: TNL's host sweep with one OpenMP thread is the sequential forward
  sweep; the device's dependency-kernel sweep evaluates every row as TNL's
  build does, so with equal iteration counts the solution is TNL's bit for
  bit (FP64 and FP32, CSR and padded layouts, relaxation 0.6 / 1.0 / 1.5);
* Jacobi: the sweeps use the library's SpMV kernels, whose row sums may be
  ordered differently from TNL's: iteration counts equal (FP64) or within one
  residue period (FP32, whose residue TNL sums in FP32), solutions within
  1e-10 (FP64) / 1e-4 (FP32) relative;
* iteration control as TNL's: residue periods 1, 3, 4 (an odd period checks
  Jacobi's x between its two sweeps), the iteration limit (exact count,
  unconverged), b = 0 (NaN residue, unconverged);
* mixed precision and a zero residue period are refused.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAYOUTS = ["CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"]


@pytest.fixture(scope="module")
def ref():
    from oracle import Reference
    R = Reference()
    threads = R.threads()
    R.set_threads(1)  # TNL's SOR sweep is sequential on one thread
    yield R
    R.set_threads(threads)


def _matrices():
    from b2s import workloads as W
    return {"poisson": W.poisson2d(20), "convdiff": W.convdiff3d(7, seed=4)}


def _solve(b2s, csr, kind, real="double", layout="CSR", omega=1.0, period=4, tol=1e-8, maxit=None, b=None):
    n = len(csr[0]) - 1
    M = b2s.SparseMatrix.from_csr(*csr[:3], csr[3], segments=layout, real=real)
    s = getattr(b2s, kind)()
    s.setMatrix(M)
    s.setOmega(omega)
    s.setResiduePeriod(period)
    s.setConvergenceResidue(tol)
    if maxit is not None:
        s.setMaxIterations(maxit)
    dt = np.float64 if real == "double" else np.float32
    x = np.zeros(n, dtype=dt)
    ok = s.solve(b.astype(dt), x)
    return ok, s.getIterations(), x


def _rhs(n):
    return np.random.default_rng(5).uniform(-1, 1, n)


@pytest.mark.parametrize("name", ["poisson", "convdiff"])
@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("omega", [0.6, 1.0, 1.5])
def test_sor_vs_tnl(b2s_lib, cuda, ref, name, real, omega):
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    b = _rhs(n)
    if real == "f32":
        b = b.astype(np.float32).astype(np.float64)
    tol = 1e-8 if real == "f64" else 1e-5
    want = ref.solve_stationary("sor", csr, b, rtol=tol, omega=omega, period=4, real=real)
    ok, it, x = _solve(b2s_lib, csr, "SOR", "double" if real == "f64" else "float", omega=omega, tol=tol, b=b)
    assert ok == want["converged"]
    if real == "f64" or it == want["iterations"]:
        assert it == want["iterations"]
        assert np.array_equal(x.astype(np.float64), want["x"]), np.max(np.abs(x - want["x"]))
    else:
        assert abs(it - want["iterations"]) <= 4
        assert np.max(np.abs(x - want["x"])) <= 1e-4 * np.max(np.abs(want["x"]))


@pytest.mark.parametrize("layout", LAYOUTS[1:])
def test_sor_padded_layouts_equal_csr(b2s_lib, cuda, layout):
    csr = _matrices()["convdiff"]
    b = _rhs(len(csr[0]) - 1)
    ok0, it0, x0 = _solve(b2s_lib, csr, "SOR", b=b, omega=1.2)
    ok1, it1, x1 = _solve(b2s_lib, csr, "SOR", layout=layout, b=b, omega=1.2)
    assert ok0 and ok1 and it0 == it1
    assert np.array_equal(x0, x1)


@pytest.mark.parametrize("name", ["poisson", "convdiff"])
@pytest.mark.parametrize("real", ["f64", "f32"])
@pytest.mark.parametrize("omega", [0.7, 1.0])
def test_jacobi_vs_tnl(b2s_lib, cuda, ref, name, real, omega):
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    b = _rhs(n)
    if real == "f32":
        b = b.astype(np.float32).astype(np.float64)
    tol = 1e-7 if real == "f64" else 1e-5
    want = ref.solve_stationary("jacobi", csr, b, rtol=tol, omega=omega, period=4, real=real)
    ok, it, x = _solve(b2s_lib, csr, "Jacobi", "double" if real == "f64" else "float", omega=omega, tol=tol, b=b)
    assert ok == want["converged"]
    rel = np.max(np.abs(x - want["x"])) / np.max(np.abs(want["x"]))
    if real == "f64":
        assert it == want["iterations"]
        assert rel <= 1e-10
    else:
        assert abs(it - want["iterations"]) <= 4
        assert rel <= 1e-4


@pytest.mark.parametrize("kind", ["Jacobi", "SOR"])
@pytest.mark.parametrize("period", [1, 3, 4])
@pytest.mark.parametrize("layout", ["CSR", "SlicedEllpack"])
def test_residue_periods_and_iteration_limit(b2s_lib, cuda, ref, kind, period, layout):
    csr = _matrices()["convdiff"]
    n = len(csr[0]) - 1
    b = _rhs(n)
    want = ref.solve_stationary(kind.lower(), csr, b, rtol=1e-8, omega=0.9, period=period)
    ok, it, x = _solve(b2s_lib, csr, kind, layout=layout, omega=0.9, period=period, b=b)
    assert ok == want["converged"] and it == want["iterations"]
    assert np.max(np.abs(x - want["x"])) <= 1e-10 * np.max(np.abs(want["x"]))
    # stopped by the iteration limit: TNL's count, unconverged, TNL's iterate
    want = ref.solve_stationary(kind.lower(), csr, b, rtol=1e-14, maxit=9, omega=0.9, period=period)
    ok, it, x = _solve(b2s_lib, csr, kind, layout=layout, omega=0.9, period=period, tol=1e-14, maxit=9, b=b)
    assert not ok and not want["converged"]
    assert it == want["iterations"]
    assert np.max(np.abs(x - want["x"])) <= 1e-12 * np.max(np.abs(want["x"]))


@pytest.mark.parametrize("kind", ["Jacobi", "SOR"])
def test_zero_rhs_and_refusals(b2s_lib, cuda, ref, kind):
    csr = _matrices()["poisson"]
    n = len(csr[0]) - 1
    want = ref.solve_stationary(kind.lower(), csr, np.zeros(n), rtol=1e-8)
    ok, it, x = _solve(b2s_lib, csr, kind, b=np.zeros(n))
    assert not ok and not want["converged"]
    assert it == want["iterations"]
    assert not np.any(x)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = getattr(b2s_lib, kind)()
    s.setMatrix(M)
    s.setResiduePeriod(0)
    with pytest.raises(b2s_lib.B2SError) as e:
        s.solve(np.ones(n), np.zeros(n))
    assert e.value.status == b2s_lib.INVALID_ARG
    s = getattr(b2s_lib, kind)()
    s.setMatrix(M)
    s.setPrecision(True)
    with pytest.raises(b2s_lib.B2SError) as e:
        s.solve(np.ones(n), np.zeros(n))
    assert e.value.status == b2s_lib.UNSUPPORTED


def test_sor_symmetric_matrix_and_cpp_setup_keys(b2s_lib, cuda, ref):
    """A SymmetricMatrix sweeps its general form; TNL's configuration keys set omega / period."""
    csr = _matrices()["poisson"]
    off, col, val, n = csr
    rows = np.repeat(np.arange(n), np.diff(off))
    keep = col <= rows
    loff = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=n))]).astype(np.int32)
    b = _rhs(n)
    want = ref.solve_stationary("sor", csr, b, rtol=1e-8, omega=1.3, period=2)
    M = b2s_lib.SparseMatrix.from_csr(loff, col[keep], val[keep], n, symmetric=True)
    s = b2s_lib.SOR()
    s.setMatrix(M)
    assert s.setup({"sor-omega": 1.3, "residue-period": 2, "convergence-residue": 1e-8})
    x = np.zeros(n)
    assert s.solve(b, x)
    assert s.getIterations() == want["iterations"]
    assert np.array_equal(x, want["x"])
