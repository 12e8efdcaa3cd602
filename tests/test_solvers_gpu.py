"""GPU parity of the Krylov solvers (through the C ABI) against TNL's own
Devices::Host runs (tests/golden/solvers.npz) and the oracle.

Criteria (TNL's reductions are order-dependent, so bits cannot match):
converged flag equal, iteration count within max(2, 2%), and
||x - x_TNL||_inf / ||x_TNL||_inf <= 1e-8 at convergence residue 1e-10.
"""
import numpy as np
import pytest

import fixtures as F

pytestmark = pytest.mark.gpu

SOLVERS = {"cg": "CG", "bicgstab": "BICGStab", "gmres": "GMRES", "tfqmr": "TFQMR", "bicgstabl": "BICGStabL"}


def solver_for(b2s, case_solver, M, precond, variant="MGSR", rmin=30, rmax=30, tol=1e-10, **extra):
    s = getattr(b2s, SOLVERS[case_solver])()
    s.setMatrix(M)
    s.setPreconditioner("diagonal" if precond else None)
    s.setConvergenceResidue(tol)
    s.setup({"gmres-variant": variant, "gmres-restarting-min": rmin, "gmres-restarting-max": rmax, **extra})
    return s


@pytest.mark.parametrize("case", F.solver_cases(), ids=lambda c: c["key"])
def test_solver_vs_tnl(b2s_lib, cuda, case):
    off, col, val, nc = F.csr(case["matrix"])
    M = b2s_lib.SparseMatrix.from_csr(off, col, val, nc)
    s = solver_for(b2s_lib, case["solver"], M, case["precond"], case["variant"], case["restart_min"],
                   case["restart_max"], **{"bicgstab-ell": case["ell"]})
    x = np.zeros(len(off) - 1)
    ok = s.solve(case["b"].copy(), x)
    assert ok == case["converged"]
    assert abs(s.getIterations() - case["iterations"]) <= max(2, 0.02 * case["iterations"])
    err = np.max(np.abs(x - case["x"])) / np.max(np.abs(case["x"]))
    assert err <= 1e-8
    assert s.report.true_residual <= 1e-9


@pytest.mark.parametrize("fmt", ["Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack"])
@pytest.mark.parametrize("solver", ["cg", "bicgstab", "gmres"])
def test_solvers_over_every_layout(b2s_lib, cuda, oracle, fmt, solver):
    from b2s import workloads as W
    csr = W.poisson2d(24, 20) if solver == "cg" else W.convdiff3d(7)
    n = len(csr[0]) - 1
    b = W.uniform(n, 5)
    ref = oracle.solve(solver, csr, b, rtol=1e-10, gmres_variant="CGSR", restart_min=30, restart_max=30)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], segments=fmt)
    s = solver_for(b2s_lib, solver, M, False, "CGSR")
    x = cuda.zeros(n, dtype=cuda.float64, device="cuda")
    assert s.solve(cuda.tensor(b, device="cuda"), x)
    assert abs(s.getIterations() - ref["iterations"]) <= max(2, 0.02 * ref["iterations"])
    assert np.max(np.abs(x.cpu().numpy() - ref["x"])) / np.max(np.abs(ref["x"])) <= 1e-8


@pytest.mark.parametrize("variant", ["CGS", "CGSR", "MGS", "MGSR"])
@pytest.mark.parametrize("restart", [(10, 30), (30, 30), (5, 5)])
def test_gmres_variants_vs_oracle(b2s_lib, cuda, oracle, variant, restart):
    from b2s import workloads as W
    csr = W.convdiff3d(8, seed=6)
    n = len(csr[0]) - 1
    b = W.uniform(n, 7)
    ref = oracle.solve("gmres", csr, b, rtol=1e-10, gmres_variant=variant, restart_min=restart[0],
                       restart_max=restart[1])
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = solver_for(b2s_lib, "gmres", M, False, variant, *restart)
    x = np.zeros(n)
    assert s.solve(b, x) == ref["converged"]
    tol_it = max(2, 0.05 * ref["iterations"]) if variant in ("CGS", "MGS") else max(2, 0.02 * ref["iterations"])
    assert abs(s.getIterations() - ref["iterations"]) <= tol_it
    assert np.max(np.abs(x - ref["x"])) / np.max(np.abs(ref["x"])) <= 1e-8


def test_max_iterations_and_nan(b2s_lib, cuda):
    from b2s import workloads as W
    csr = W.poisson2d(32)
    n = len(csr[0]) - 1
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = solver_for(b2s_lib, "cg", M, False)
    s.setMaxIterations(5)
    x = np.zeros(n)
    assert not s.solve(np.ones(n), x)
    assert s.report.status == b2s_lib.NOT_CONVERGED
    b = np.ones(n)
    b[3] = np.nan  # a poisoned right-hand side ends as a NaN residue, not a hang
    s2 = solver_for(b2s_lib, "bicgstab", M, False)
    assert not s2.solve(b, np.zeros(n))
    assert s2.report.status == b2s_lib.NAN


def test_zero_rhs_and_exact_initial_guess(b2s_lib, cuda):
    from b2s import workloads as W
    csr = W.poisson2d(10)
    n = len(csr[0]) - 1
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    for solver in SOLVERS:
        s = solver_for(b2s_lib, solver, M, False)
        x = np.zeros(n)
        assert s.solve(np.zeros(n), x)
        assert np.all(x == 0)


@pytest.mark.parametrize("solver,maker", [("cg", "diffusion"), ("bicgstab", "convdiff"), ("gmres", "convdiff")])
@pytest.mark.parametrize("precond", [False, True])
def test_mixed_precision_reaches_fp64_tolerance(b2s_lib, cuda, oracle, solver, maker, precond):
    from b2s import workloads as W
    csr = W.diffusion3d(20, seed=3) if maker == "diffusion" else W.convdiff3d(16, seed=4)
    n = len(csr[0]) - 1
    b = W.uniform(n, 9)
    ref = oracle.solve(solver, csr, b, rtol=1e-12, precond=precond, gmres_variant="CGSR", restart_min=30,
                       restart_max=30)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = solver_for(b2s_lib, solver, M, precond, "CGSR")
    s.setPrecision(True)
    x = np.zeros(n)
    assert s.solve(b, x)
    assert s.report.true_residual <= 1e-10
    assert s.report.refinements >= 1
    # error against the FP64 oracle solution
    assert np.max(np.abs(x - ref["x"])) / np.max(np.abs(ref["x"])) <= 1e-7


def test_fp32_plain_solve(b2s_lib, cuda):
    from b2s import workloads as W
    csr = W.poisson2d(30)
    n = len(csr[0]) - 1
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], real="float")
    s = solver_for(b2s_lib, "cg", M, False, tol=1e-5)
    x = np.zeros(n, dtype=np.float32)
    assert s.solve(np.ones(n, dtype=np.float32), x)
    assert s.report.true_residual <= 1e-4


def test_repeated_solves_reuse_state(b2s_lib, cuda):
    """The same solver object solves several right-hand sides (graphs are reused)."""
    from b2s import workloads as W
    csr = W.poisson2d(40)
    n = len(csr[0]) - 1
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = solver_for(b2s_lib, "cg", M, True)
    first = None
    for k in range(3):
        b = W.uniform(n, 20 + (k % 2))
        x = np.zeros(n)
        assert s.solve(b, x)
        if k == 0:
            first = (x.copy(), s.getIterations())
        if k == 2:
            assert np.array_equal(x, first[0]) and s.getIterations() == first[1]


@pytest.mark.parametrize("solver,maker,slack", [("cg", "diffusion", 1.15), ("bicgstab", "convdiff", 1.3),
                                                ("gmres", "convdiff", 1.15)])
def test_mixed_precision_keeps_the_iteration_count(b2s_lib, cuda, solver, maker, slack):
    """Reliable updates (CG, BiCGStab) keep the FP32 recurrence across the FP64
    residual replacements, and GMRES refines once per restart cycle, so the
    mixed solve needs about as many iterations as the FP64 one."""
    from b2s import workloads as W
    csr = W.diffusion3d(32, seed=3) if maker == "diffusion" else W.convdiff3d(32, seed=4)
    n = len(csr[0]) - 1
    b = W.uniform(n, 9)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], keep_fp32_copy=True)
    its = {}
    for mixed in (False, True):
        s = solver_for(b2s_lib, solver, M, False, "CGSR", tol=1e-10)
        s.setPrecision(mixed)
        x = np.zeros(n)
        assert s.solve(b, x)
        assert s.report.true_residual <= (1e-10 if mixed else 2e-10)
        its[mixed] = s.getIterations()
    assert its[True] <= slack * its[False] + 10, its


@pytest.mark.parametrize("name,pre", [("convdiff", 0), ("convdiff", 1), ("convdiff", 2), ("poisson", 0),
                                      ("random", 1)])
@pytest.mark.parametrize("restart", [(30, 30), (10, 30)])
def test_gmres_cwy_vs_tnl(b2s_lib, cuda, name, pre, restart):
    """GMRES with Householder reflections in compact WY form against TNL's own
    (GMRES.hpp:348-715): converged flag, solution within 1e-8 at residue 1e-10
    (1e-4 with ILU(0), see below), and the iteration count inside the range TNL
    itself gives on 1 to 16 OpenMP threads and on all the host's cores, widened
    by max(2, 2 %) (with Jacobi on the convection-diffusion matrix TNL took 55
    iterations on an 8-core host and 62 on a 16-core one). The solution is
    compared with TNL's 4-thread run: with all 16 cores TNL's CWY with ILU(0)
    once ended 6e-5 away from it, and that 4-thread run itself moves between
    hosts by a few 1e-6, so with ILU(0) the bound is TNL's own spread."""
    from oracle import Reference
    from b2s import workloads as W
    R = Reference()
    g = np.random.default_rng(8)
    n = 2000
    lens = g.integers(1, 10, n)
    rows = [np.unique(np.concatenate([[i], g.choice(n, L, replace=False)])) for i, L in enumerate(lens)]
    off = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    col = np.concatenate(rows).astype(np.int32)
    val = g.uniform(-1, 1, len(col))
    val[col == np.repeat(np.arange(n), np.diff(off))] = 12.0
    csr = {"convdiff": W.convdiff3d(12, seed=4), "poisson": W.poisson2d(40), "random": (off, col, val, n)}[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(3).uniform(-1, 1, n)
    kw = dict(rtol=1e-10, precond=pre, gmres_variant="CWY", restart_min=restart[0], restart_max=restart[1])
    its = [R.solve("gmres", csr, b, **kw)["iterations"]]  # all the host's cores
    base = R.lib.tnlref_get_threads()
    try:
        for th in (1, 2, 4, 8, 16):
            R.lib.tnlref_set_threads(th)
            r = R.solve("gmres", csr, b, **kw)
            its.append(r["iterations"])
            if th == 4:  # the solution compared against: the same on every host
                want = r
    finally:
        R.lib.tnlref_set_threads(base)
    lo, hi = min(its), max(its)
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    s = b2s_lib.GMRES()
    s.setMatrix(M)
    s.setPreconditioner({0: None, 1: "diagonal", 2: "ilu0"}[pre])
    s.setConvergenceResidue(1e-10)
    s.setup({"gmres-variant": "CWY", "gmres-restarting-min": restart[0], "gmres-restarting-max": restart[1]})
    for dev in (False, True):
        if dev:
            x = cuda.zeros(n, dtype=cuda.float64, device="cuda")
            ok = s.solve(cuda.tensor(b, device="cuda"), x)
            x = x.cpu().numpy()
        else:
            x = np.zeros(n)
            ok = s.solve(b, x)
        assert ok == want["converged"]
        tol = max(2, 0.02 * hi)
        assert lo - tol <= s.getIterations() <= hi + tol, (s.getIterations(), its)
        assert np.max(np.abs(x - want["x"])) / np.max(np.abs(want["x"])) <= (1e-4 if pre == 2 else 1e-8)
