"""The distributed SpMV and solvers on one GPU.

Several ranks run as threads of this process (LocalGroup: host barriers between
their steps, exchanges as device copies; no kernel waits on another), each with
its own rows, halo plan and kernels; a world_size-1 NCCL process group runs the
torch.distributed path itself.

* the distributed product equals the single-matrix product bit for bit with
  the CSR scalar kernel (each row keeps its element order, one thread sums it),
  and for the 7-point Laplacian with the default kernel too; the default
  kernel on long irregular rows (its summation form depends on where a row
  falls among the nonzero windows, which moves with the local offsets), other
  layouts and the overlapped (owned block + ghost block) product within 1e-14;
* distributed CG, BiCGStab, TFQMR and GMRES (TNL's recurrences with
  all-reduced dots) reach the single-GPU solvers' solutions (1e-8) in as many
  iterations (max(2, 5 %)), without and with Jacobi; block ILU(0) converges and
  on one rank equals the single-GPU ILU(0) solve;
* against TNL's own solvers (Devices::Host, compiled from the reference
  headers): every solver and the four Gram-Schmidt variants of GMRES, with the
  adaptive restart length, reach TNL's solution (1e-7) in as many iterations
  (max(2, 5 %)); GMRES stopped by the iteration limit stops where TNL's does,
  unconverged, at TNL's iterate.
"""
import os
import socket
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_ranks(world, fn, timeout=300):
    from b2s.distributed import LocalGroup
    groups = LocalGroup.world(world, timeout=timeout)
    res, errs = {}, []

    def run(g):
        try:
            res[g.rank] = fn(g)
        except BaseException as e:  # noqa: BLE001 - reported below
            errs.append(e)
            g._w.barrier.abort()

    ts = [threading.Thread(target=run, args=(g,)) for g in groups]
    for t in ts:
        t.start()
    for t in ts:
        t.join(timeout + 60)
    assert not errs, errs
    return res


def _local_rows(csr, lo, hi):
    off, col, val, _ = csr
    return (off[lo:hi + 1] - off[lo]).astype(np.int32), col[off[lo]:off[hi]], val[off[lo]:off[hi]]


def _matrices():
    from b2s import workloads as W
    return {"irregular": W.irregular(5000, seed=12, mu=np.log(10), sigma=1.0, hi=300),
            "laplace3d": W.laplace3d(20), "convdiff": W.convdiff3d(14, seed=5),
            "diffusion": W.diffusion3d(16, seed=3)}


@pytest.mark.parametrize("name", ["irregular", "laplace3d"])
@pytest.mark.parametrize("world", [2, 3, 4])
def test_product_bitwise(b2s_lib, cuda, name, world):
    from b2s.distributed import DistributedMatrix, split_range
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    x = np.random.default_rng(2).uniform(-1, 1, n)
    xg = cuda.tensor(x, device="cuda")
    want = {}
    for kern in ("CSRScalar", "CSRDefault"):
        G = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], csr_kernel=kern)
        yg = cuda.zeros(n, dtype=cuda.float64, device="cuda")
        G.vectorProduct(xg, yg)
        want[kern] = yg.cpu().numpy()
    cases = (("CSR", False, "CSRScalar"), ("CSR", False, "CSRDefault"), ("CSR", True, "CSRDefault"),
             ("SlicedEllpack", False, "CSRDefault"), ("BiEllpack", True, "CSRDefault"))

    def fn(g):
        lo, hi = split_range(n, g.rank, g.size)
        out = {}
        for seg, overlap, kern in cases:
            A = DistributedMatrix(g, *_local_rows(csr, lo, hi), n, n, segments=seg, overlap=overlap,
                                  csr_kernel=kern)
            v = A.vector("cuda")
            v.getLocalView().copy_(xg[lo:hi])
            y = cuda.zeros(hi - lo, dtype=cuda.float64, device="cuda")
            A.vectorProduct(v, y)
            out[(seg, overlap, kern)] = (lo, hi, y.cpu().numpy())
        return out

    res = _run_ranks(world, fn)
    for key in res[0]:
        got = np.zeros(n)
        for r in range(world):
            lo, hi, y = res[r][key]
            got[lo:hi] = y
        w = want[key[2]]
        if key == ("CSR", False, "CSRScalar") or (key == ("CSR", False, "CSRDefault") and name == "laplace3d"):
            assert np.array_equal(got, w), key
        else:
            assert np.max(np.abs(got - w)) <= 1e-14 * np.max(np.abs(w)), key


SOLVERS = {"cg": ("CG", "CG"), "bicgstab": ("BICGStab", "BICGStab"), "tfqmr": ("TFQMR", "TFQMR"),
           "gmres": ("GMRES", "GMRES")}


@pytest.mark.parametrize("kind,name", [("cg", "diffusion"), ("bicgstab", "convdiff"), ("tfqmr", "convdiff"),
                                       ("cg", "laplace3d"), ("gmres", "convdiff")])
@pytest.mark.parametrize("pre", [None, "diagonal"])
@pytest.mark.parametrize("world", [1, 3])
def test_solvers_vs_single_gpu(b2s_lib, cuda, kind, name, pre, world):
    import b2s.distributed as D
    from b2s.distributed import DistributedMatrix, split_range
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(4).uniform(-1, 1, n)
    S = getattr(b2s_lib, SOLVERS[kind][0])()
    S.setMatrix(b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3]))
    S.setPreconditioner(pre)
    S.setConvergenceResidue(1e-10)
    xs = np.zeros(n)
    assert S.solve(b, xs)
    bg = cuda.tensor(b, device="cuda")

    def fn(g):
        lo, hi = split_range(n, g.rank, g.size)
        A = DistributedMatrix(g, *_local_rows(csr, lo, hi), n, n, overlap=(g.rank % 2 == 1))
        s = getattr(D, SOLVERS[kind][1])(A, preconditioner=pre, convergence_residue=1e-10)
        x = A.vector("cuda")
        ok = s.solve(bg[lo:hi].clone(), x)
        return lo, hi, ok, s.iterations, x.getLocalView().cpu().numpy()

    res = _run_ranks(world, fn)
    x = np.zeros(n)
    its = {res[r][3] for r in range(world)}
    assert len(its) == 1, its  # every rank took the same decisions
    for r in range(world):
        lo, hi, ok, it, xl = res[r]
        assert ok
        x[lo:hi] = xl
    it = its.pop()
    assert abs(it - S.getIterations()) <= max(2, 0.05 * S.getIterations()), (it, S.getIterations())
    assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) <= 1e-8


def _gather_solution(res, world, n):
    x = np.zeros(n)
    for r in range(world):
        lo, hi, ok, it, xl = res[r]
        x[lo:hi] = xl
    its = {res[r][3] for r in range(world)}
    oks = {res[r][2] for r in range(world)}
    assert len(its) == 1 and len(oks) == 1, (its, oks)  # every rank took the same decisions
    return x, its.pop(), oks.pop()


TNL_CASES = [("cg", "diffusion", {}), ("bicgstab", "convdiff", {}), ("tfqmr", "convdiff", {}),
             ("gmres", "convdiff", {"variant": "CGS"}), ("gmres", "convdiff", {"variant": "CGSR"}),
             ("gmres", "convdiff", {"variant": "MGS"}),
             ("gmres", "convdiff", {"variant": "MGSR", "restarting_min": 10, "restarting_max": 30}),
             ("gmres", "diffusion", {"variant": "CGSR", "restarting_min": 5, "restarting_max": 20})]


@pytest.mark.parametrize("case", range(len(TNL_CASES)))
@pytest.mark.parametrize("pre", [None, "diagonal"])
def test_distributed_solvers_vs_tnl(b2s_lib, cuda, case, pre):
    import b2s.distributed as D
    from b2s.distributed import DistributedMatrix, split_range
    from oracle import Reference
    kind, name, kw = TNL_CASES[case]
    csr = _matrices()[name]
    n = len(csr[0]) - 1
    b = np.random.default_rng(9).uniform(-1, 1, n)
    gm = {"gmres_variant": kw.get("variant", "MGSR"), "restart_min": kw.get("restarting_min", 10),
          "restart_max": kw.get("restarting_max", 10)}
    want = Reference().solve(kind, csr, b, rtol=1e-10, precond=1 if pre else 0, **gm)
    assert want["converged"]
    bg = cuda.tensor(b, device="cuda")
    world = 3

    def fn(g):
        lo, hi = split_range(n, g.rank, g.size)
        A = DistributedMatrix(g, *_local_rows(csr, lo, hi), n, n, overlap=(g.rank == 1))
        s = getattr(D, SOLVERS[kind][1])(A, preconditioner=pre, convergence_residue=1e-10, **kw)
        x = A.vector("cuda")
        ok = s.solve(bg[lo:hi].clone(), x)
        return lo, hi, ok, s.iterations, x.getLocalView().cpu().numpy()

    x, it, ok = _gather_solution(_run_ranks(world, fn), world, n)
    assert ok
    assert abs(it - want["iterations"]) <= max(2, 0.05 * want["iterations"]), (it, want["iterations"])
    assert np.max(np.abs(x - want["x"])) / np.max(np.abs(want["x"])) <= 1e-7


@pytest.mark.parametrize("variant", ["CGS", "MGSR"])
def test_distributed_gmres_stops_at_the_iteration_limit(b2s_lib, cuda, variant):
    import b2s.distributed as D
    from b2s.distributed import DistributedMatrix, split_range
    from oracle import Reference
    csr = _matrices()["convdiff"]
    n = len(csr[0]) - 1
    b = np.random.default_rng(10).uniform(-1, 1, n)
    maxit = 13  # inside the second restart cycle of length 10
    want = Reference().solve("gmres", csr, b, rtol=1e-14, maxit=maxit, gmres_variant=variant, restart_min=10,
                             restart_max=10)
    assert not want["converged"]
    bg = cuda.tensor(b, device="cuda")

    def fn(g):
        lo, hi = split_range(n, g.rank, g.size)
        A = DistributedMatrix(g, *_local_rows(csr, lo, hi), n, n)
        s = D.GMRES(A, variant=variant, convergence_residue=1e-14, max_iterations=maxit)
        x = A.vector("cuda")
        ok = s.solve(bg[lo:hi].clone(), x)
        return lo, hi, ok, s.iterations, x.getLocalView().cpu().numpy()

    x, it, ok = _gather_solution(_run_ranks(2, fn), 2, n)
    assert not ok
    assert it == want["iterations"], (it, want["iterations"])
    assert np.max(np.abs(x - want["x"])) / np.max(np.abs(want["x"])) <= 1e-10


def test_block_ilu0(b2s_lib, cuda):
    import b2s.distributed as D
    from b2s.distributed import DistributedMatrix, split_range
    csr = _matrices()["convdiff"]
    n = len(csr[0]) - 1
    b = np.random.default_rng(6).uniform(-1, 1, n)
    bg = cuda.tensor(b, device="cuda")
    S = b2s_lib.BICGStab()
    S.setMatrix(b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3]))
    S.setPreconditioner("ilu0")
    S.setConvergenceResidue(1e-10)
    xs = np.zeros(n)
    assert S.solve(b, xs)
    for world in (1, 4):
        def fn(g):
            lo, hi = split_range(n, g.rank, g.size)
            A = DistributedMatrix(g, *_local_rows(csr, lo, hi), n, n)
            s = D.BICGStab(A, preconditioner="ilu0", convergence_residue=1e-10)
            x = A.vector("cuda")
            ok = s.solve(bg[lo:hi].clone(), x)
            return lo, hi, ok, s.iterations, x.getLocalView().cpu().numpy()

        res = _run_ranks(world, fn)
        x = np.zeros(n)
        for r in range(world):
            lo, hi, ok, it, xl = res[r]
            assert ok
            x[lo:hi] = xl
        assert np.max(np.abs(x - xs)) / np.max(np.abs(xs)) <= 1e-8
        if world == 1:  # one block: the global ILU(0)
            assert abs(res[0][3] - S.getIterations()) <= 2


def test_torch_distributed_nccl_single_rank(b2s_lib, cuda):
    """The torch.distributed path (NCCL, one rank): product and CG."""
    import torch.distributed as dist
    from datetime import timedelta
    import b2s.distributed as D
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    cuda.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        g = D.TorchGroup()
        csr = _matrices()["diffusion"]
        n = len(csr[0]) - 1
        A = D.DistributedMatrix(g, *csr[:3], n, n)
        x = np.random.default_rng(1).uniform(-1, 1, n)
        v = A.vector("cuda")
        v.getLocalView().copy_(cuda.tensor(x, device="cuda"))
        y = cuda.zeros(n, dtype=cuda.float64, device="cuda")
        A.vectorProduct(v, y)
        G = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
        yg = np.zeros(n)
        G.vectorProduct(x, yg)
        assert np.array_equal(y.cpu().numpy(), yg)
        s = D.CG(A, preconditioner="diagonal", convergence_residue=1e-10)
        xs = A.vector("cuda")
        assert s.solve(cuda.tensor(np.ones(n), device="cuda"), xs)
    finally:
        dist.destroy_process_group()
