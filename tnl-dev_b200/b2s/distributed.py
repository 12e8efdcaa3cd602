"""Row-block distributed SpMV and Krylov solvers across GPUs.

TNL's model (Matrices/DistributedMatrix.h, DistributedMatrix_impl.h:202-245):
every rank owns a contiguous range of rows (Containers/Partitioner.h:30-72,
``split_range``) and stores them as a local matrix; the input vector is a
DistributedVector whose local storage is [owned entries | ghosts]
(Containers/DistributedArrayView.hpp:174-200), the ghosts are brought in by a
synchronizer, and the product is the local matrix times that storage. TNL's
linear solvers run unchanged on such matrices and vectors, with every dot
product becoming an all-reduce.

Here:
* ``HaloPlan`` is the synchronizer, built from the local matrix's column
  indices: the ghosts are exactly the off-rank columns the rows reference
  (sorted, hence grouped by owner); each owner learns once which of its entries
  to send. The local matrix's columns are renumbered to [owned | ghosts] (the
  order of the elements inside a row is kept, so row sums keep their order).
* ``DistributedVector.startSynchronization`` packs the entries to send with
  the library's gather kernel and posts point-to-point sends and receives
  straight into the ghost part of the local storage;
  ``waitForSynchronization`` completes them.
* ``DistributedMatrix.vectorProduct`` exchanges, then multiplies. With
  ``overlap=True`` the local matrix is split into the owned-column block and
  the ghost-column block: the owned block's product runs while the halo is in
  flight, the ghost block is added after it arrives (sums are then split, so
  results differ from the single product by rounding only).
* ``CG``, ``BICGStab``, ``TFQMR`` and ``GMRES`` follow TNL's recurrences
  (CG.hpp:11-104, BICGStab.hpp:33-145, TFQMR.hpp:18-114, GMRES.hpp:76-760)
  with local device kernels and one all-reduce per dot product (TNL reduces
  every dot over MPI the same way); classical Gram-Schmidt reduces all of a
  step's projections in one all-reduce.

Communication goes through a group object: ``TorchGroup`` wraps a
torch.distributed process group (NCCL between GPUs, one process per GPU;
gloo for host tensors), ``LocalGroup`` runs several ranks as threads of one
process (host barriers between steps, exchanges as copies) so the whole path
can be exercised on a single device.
"""
from __future__ import annotations

import threading

import numpy as np

# ---------------------------------------------------------------------------
# Containers::Partitioner (Partitioner.h:30-72)


def split_range(global_size: int, rank: int, nproc: int) -> tuple[int, int]:
    """splitRange: [min(n, r n / p), min(n, (r + 1) n / p))."""
    return (min(global_size, rank * global_size // nproc), min(global_size, (rank + 1) * global_size // nproc))


def get_offset(global_size: int, rank: int, nproc: int) -> int:
    return rank * global_size // nproc


def get_owner(i, global_size: int, nproc: int):
    """getOwner (vectorised): the rank whose range holds global index i. TNL's
    formula (i p / n, bumped once) is exact for n >= p; this is the first rank
    whose range ends above i, which agrees with it there and also holds when
    some ranks own nothing."""
    i = np.asarray(i, dtype=np.int64)
    ends = np.array([min(global_size, (r + 1) * global_size // nproc) for r in range(nproc)], dtype=np.int64)
    return np.searchsorted(ends, i, side="right").astype(np.int64)


# ---------------------------------------------------------------------------
# Groups


class TorchGroup:
    """torch.distributed process group (the default one unless `group` is given)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self._d = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def allgather_obj(self, obj):
        out = [None] * self.size
        self._d.all_gather_object(out, obj, group=self.group)
        return out

    def start_exchange(self, sends: dict, recvs: dict):
        """Post sends[q] -> rank q and recvs[q] <- rank q; returns the pending requests."""
        d = self._d
        ops = []
        glob = (lambda q: d.get_global_rank(self.group, q)) if self.group is not None else (lambda q: q)
        for q, t in recvs.items():
            ops.append(d.P2POp(d.irecv, t, glob(q), group=self.group))
        for q, t in sends.items():
            ops.append(d.P2POp(d.isend, t, glob(q), group=self.group))
        return d.batch_isend_irecv(ops) if ops else []

    def wait(self, reqs):
        for r in reqs:
            r.wait()

    def allreduce_sum(self, t):
        self._d.all_reduce(t, op=self._d.ReduceOp.SUM, group=self.group)

    def barrier(self):
        self._d.barrier(group=self.group)


class _LocalWorld:
    def __init__(self, size: int, timeout: float):
        self.size = size
        self.barrier = threading.Barrier(size, timeout=timeout)
        self.slots = [None] * size
        self.mail = {}


class LocalGroup:
    """One of `size` ranks run as threads of this process (see ``LocalGroup.world``).
    Collective calls block on a host barrier (bounded by `timeout` seconds); device
    data moves by copies on the current stream, so no kernel waits on another."""

    @staticmethod
    def world(size: int, timeout: float = 120.0):
        w = _LocalWorld(size, timeout)
        return [LocalGroup(w, r) for r in range(size)]

    def __init__(self, world: _LocalWorld, rank: int):
        self._w = world
        self.rank = rank
        self.size = world.size

    def allgather_obj(self, obj):
        w = self._w
        w.slots[self.rank] = obj
        w.barrier.wait()
        out = list(w.slots)
        w.barrier.wait()
        return out

    def start_exchange(self, sends: dict, recvs: dict):
        w = self._w
        for q, t in sends.items():
            w.mail[(self.rank, q)] = t
        w.barrier.wait()
        for q, t in recvs.items():
            t.copy_(w.mail.pop((q, self.rank)))
        return [None]

    def wait(self, reqs):
        if reqs:
            self._w.barrier.wait()  # the senders' buffers may be reused after this

    def allreduce_sum(self, t):
        w = self._w
        w.slots[self.rank] = t.clone()
        w.barrier.wait()
        acc = w.slots[0].clone()
        for q in range(1, self.size):  # rank order: every rank gets the same bits
            acc += w.slots[q]
        w.barrier.wait()
        t.copy_(acc)

    def barrier(self):
        self._w.barrier.wait()


# ---------------------------------------------------------------------------
# The synchronizer


class HaloPlan:
    """Ghost layout and exchange lists of one rank, from the global column
    indices its rows reference."""

    def __init__(self, group, local_range, global_size: int, columns):
        lo, hi = (int(local_range[0]), int(local_range[1]))
        cols = np.asarray(columns, dtype=np.int64)
        bad = bool(cols.size and (cols.min() < 0 or cols.max() >= global_size))
        # every rank takes the same collective steps, errors included
        info = group.allgather_obj((lo, hi, bad))
        if any(i[2] for i in info):
            raise ValueError("column index outside [0, columns) on rank(s) "
                             f"{[q for q, i in enumerate(info) if i[2]]}")
        self.local_range = (lo, hi)
        self.global_size = int(global_size)
        self.n_local = hi - lo
        off_rank = (cols < lo) | (cols >= hi)
        self.ghosts = np.unique(cols[off_rank])
        ranges = [(i[0], i[1]) for i in info]
        ok = ranges[0][0] == 0 and ranges[-1][1] == global_size
        ok = ok and all(ranges[q][0] == ranges[q - 1][1] and ranges[q][0] <= ranges[q][1] for q in range(1, len(ranges)))
        if not ok:
            raise ValueError("the ranks' row ranges must cover [0, rows) contiguously, in rank order")
        # owner of a ghost: the first rank whose range ends above it (empty ranges are passed over)
        ends = np.array([r[1] for r in ranges], dtype=np.int64)
        owner = np.searchsorted(ends, self.ghosts, side="right")
        self.recv = {}  # q -> (offset into the ghost part, count)
        requests = {}
        pos = 0
        for q in np.unique(owner):
            q = int(q)
            sel = self.ghosts[owner == q]
            self.recv[q] = (pos, len(sel))
            requests[q] = sel
            pos += len(sel)
        # every rank learns which of its entries the others need
        asked = group.allgather_obj(requests)
        self.send = {}  # q -> local indices to send to q
        for q in range(group.size):
            if q == group.rank:
                continue
            want = asked[q].get(group.rank)
            if want is not None and len(want):
                idx = np.asarray(want, dtype=np.int64) - lo
                if idx.min() < 0 or idx.max() >= self.n_local:
                    raise ValueError("a rank asked for entries this rank does not own")
                self.send[q] = idx.astype(np.int32)
        self.send_total = sum(len(v) for v in self.send.values())

    @property
    def n_ghosts(self) -> int:
        return len(self.ghosts)

    def renumber(self, columns):
        """Global column indices -> [owned | ghosts] local indices."""
        c = np.asarray(columns, dtype=np.int64)
        lo, hi = self.local_range
        out = c - lo
        g = (c < lo) | (c >= hi)
        out[g] = self.n_local + np.searchsorted(self.ghosts, c[g])
        return out.astype(np.int32)


# ---------------------------------------------------------------------------
# Containers::DistributedVector with ghosts


class DistributedVector:
    """Local storage [owned entries | ghosts] of one rank (a torch tensor on this
    rank's device, or on the host for gloo groups)."""

    def __init__(self, group, plan: HaloPlan, dtype=None, device=None, data=None):
        import torch
        self.group = group
        self.plan = plan
        n = plan.n_local + plan.n_ghosts
        if data is not None:
            if data.numel() != n:
                raise ValueError("data must hold the owned entries and the ghosts")
            self.data = data
        else:
            self.data = torch.zeros(n, dtype=dtype or torch.float64, device=device)
        self._send = None
        self._send_idx = None
        self._pending = None

    def getLocalView(self):
        return self.data[: self.plan.n_local]

    def getConstLocalViewWithGhosts(self):
        return self.data

    def getLocalRange(self):
        return self.plan.local_range

    def getSize(self):
        return self.plan.global_size

    def _buffers(self):
        import torch
        if self._send is None:
            p = self.plan
            self._send = torch.empty(max(p.send_total, 1), dtype=self.data.dtype, device=self.data.device)
            idx = np.concatenate([p.send[q] for q in sorted(p.send)]) if p.send else np.zeros(0, np.int32)
            self._send_idx = torch.tensor(idx, dtype=torch.int32, device=self.data.device)
            self._send_views, self._recv_views = {}, {}
            pos = 0
            for q in sorted(p.send):
                k = len(p.send[q])
                self._send_views[q] = self._send[pos:pos + k]
                pos += k
            for q, (o, k) in p.recv.items():
                self._recv_views[q] = self.data[p.n_local + o: p.n_local + o + k]

    def startSynchronization(self):
        """Pack the entries the other ranks reference and post the exchange."""
        self._buffers()
        p = self.plan
        if p.send_total:
            local = self.data[: p.n_local]
            if self.data.is_cuda:
                from . import gather
                gather(local, self._send_idx, self._send[: p.send_total])
            else:  # host tensors (gloo groups): the pack is plain indexing
                self._send[: p.send_total] = local[self._send_idx.long()]
        self._pending = self.group.start_exchange(self._send_views, self._recv_views)

    def waitForSynchronization(self):
        if self._pending is not None:
            self.group.wait(self._pending)
            self._pending = None

    def synchronize(self):
        self.startSynchronization()
        self.waitForSynchronization()


# ---------------------------------------------------------------------------
# Matrices::DistributedMatrix


class DistributedMatrix:
    """The rows [lo, hi) of a global matrix on this rank (CSR arrays with global
    column indices), stored in any of the library's layouts."""

    def __init__(self, group, offsets, columns, values, global_rows: int, global_cols: int, local_range=None,
                 segments: str = "CSR", real: str = "double", overlap: bool = False, **matrix_opts):
        from . import SparseMatrix
        self.group = group
        self.rows, self.cols = int(global_rows), int(global_cols)
        lr = local_range or split_range(self.rows, group.rank, group.size)
        off = np.ascontiguousarray(offsets, dtype=np.int32)
        if len(off) - 1 != lr[1] - lr[0]:
            raise ValueError("the local CSR must hold exactly the rows of the local range")
        if self.rows != self.cols:
            raise ValueError("the distributed matrix must be square (columns split as the rows)")
        col = np.asarray(columns)
        val = np.asarray(values, dtype=np.float64)
        self.plan = HaloPlan(group, lr, self.cols, col)
        lcol = self.plan.renumber(col)
        n_ext = self.plan.n_local + self.plan.n_ghosts
        self.real = real
        self.overlap = bool(overlap)
        self.segments = segments
        self._opts = matrix_opts  # SparseMatrix.from_csr options (csr_kernel, slice_size, ...)
        self._csr = (off, lcol, val)
        self.local = SparseMatrix.from_csr(off, lcol, val, max(n_ext, 1), segments=segments, real=real, **matrix_opts)
        self._diag_block = None
        if self.overlap:
            own = lcol < self.plan.n_local
            rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
            o_off = np.concatenate([[0], np.cumsum(np.bincount(rows[~own], minlength=len(off) - 1))]).astype(np.int32)
            self._diag_block = self._block(own)
            self.ghost_block = SparseMatrix.from_csr(o_off, lcol[~own] - self.plan.n_local, val[~own],
                                                     max(self.plan.n_ghosts, 1), segments="CSR", real=self.real)

    def _block(self, own):
        from . import SparseMatrix
        off, lcol, val = self._csr
        rows = np.repeat(np.arange(len(off) - 1), np.diff(off))
        d_off = np.concatenate([[0], np.cumsum(np.bincount(rows[own], minlength=len(off) - 1))]).astype(np.int32)
        return SparseMatrix.from_csr(d_off, lcol[own], val[own], max(self.plan.n_local, 1), segments=self.segments,
                                     real=self.real, **self._opts)

    def diagonal_block(self):
        """The owned-column block (n_local x n_local): the local matrix of the
        block-Jacobi preconditioners (TNL's ILU0 of a distributed matrix keeps
        the local columns only, ILU0.hpp:30-85)."""
        if self._diag_block is None:
            self._diag_block = self._block(self._csr[1] < self.plan.n_local)
        return self._diag_block

    def getRows(self):
        return self.rows

    def getColumns(self):
        return self.cols

    def getLocalRowRange(self):
        return self.plan.local_range

    def getLocalMatrix(self):
        return self.local

    def vector(self, device=None):
        """A DistributedVector laid out for this matrix's products."""
        import torch
        dt = torch.float64 if self.real == "double" else torch.float32
        return DistributedVector(self.group, self.plan, dtype=dt, device=device)

    def vectorProduct(self, inVector: DistributedVector, outLocal):
        """outLocal = A_local * [owned | ghosts] (DistributedMatrix_impl.h:216-245);
        the halo exchange runs inside the call."""
        if inVector.plan is not self.plan:
            raise ValueError("the input vector was not laid out for this matrix")
        nloc = self.plan.n_local
        if not self.overlap:
            inVector.synchronize()
            if nloc:
                self.local.vectorProduct(inVector.data, outLocal)
            return
        inVector.startSynchronization()
        if nloc:
            self._diag_block.vectorProduct(inVector.data[:nloc], outLocal)
        inVector.waitForSynchronization()
        if self.plan.n_ghosts:
            g = inVector.data[nloc:]
            self.ghost_block.vectorProduct(g, outLocal, 1.0, 1.0)


# ---------------------------------------------------------------------------
# Linear solvers over a DistributedMatrix (IterativeSolver control,
# IterativeSolver.hpp:98-146)


class _DistSolver:
    def __init__(self, matrix: DistributedMatrix, preconditioner=None, convergence_residue=1e-6,
                 max_iterations=1000000000, min_iterations=0, divergence_residue=float("inf")):
        import torch
        from . import Preconditioner
        self.A = matrix
        self.g = matrix.group
        self.tol = float(convergence_residue)
        self.maxit = int(max_iterations)
        self.minit = int(min_iterations)
        self.divtol = float(divergence_residue)
        if preconditioner not in (None, "", "none", "diagonal", "jacobi", "ilu0"):
            raise ValueError("distributed solvers take no preconditioner, Jacobi (diagonal) or block ILU(0)")
        self.pre = None
        if preconditioner in ("diagonal", "jacobi", "ilu0") and matrix.plan.n_local:
            self.pre = Preconditioner(matrix.diagonal_block(), "ilu0" if preconditioner == "ilu0" else "diagonal")
        self._has_pre = preconditioner in ("diagonal", "jacobi", "ilu0")
        self._acc = torch.zeros(1, dtype=torch.float64, device=self._device())
        self.iterations = 0
        self.residue = float("nan")

    def _device(self):
        return "cuda"

    # ( a, b ) over all ranks: the local dot on the device, then the all-reduce
    def dot(self, a, b) -> float:
        from . import dot
        dot(a, b, self._acc)
        self.g.allreduce_sum(self._acc)
        return float(self._acc.item())

    def norm(self, a) -> float:
        return float(np.sqrt(self.dot(a, a)))

    def precond(self, src, dst):
        if self.pre is not None:  # a rank without rows has nothing to precondition
            self.pre.solve(src, dst)

    def check_next(self) -> bool:
        r = self.residue
        return not (np.isnan(r) or self.iterations > self.maxit or (r > self.divtol and self.iterations >= self.minit)
                    or (r < self.tol and self.iterations >= self.minit))

    def next_iteration(self) -> bool:
        go = self.check_next()
        self.iterations += 1
        return go

    def converged(self) -> bool:
        r = self.residue
        if np.isnan(r):
            return False
        if r > self.divtol and self.iterations > self.minit:
            return False
        if self.iterations >= self.maxit:
            return False
        return r <= self.tol

    def _local(self, n):
        import torch
        dt = torch.float64 if self.A.real == "double" else torch.float32
        return torch.zeros(n, dtype=dt, device=self._device())


class CG(_DistSolver):
    """Solvers::Linear::CG over a DistributedMatrix (CG.hpp:11-104)."""

    def solve(self, b, x: DistributedVector) -> bool:
        from . import axpby
        A = self.A
        n = A.plan.n_local
        xl = x.getLocalView()
        r, z, Ap = self._local(n), self._local(n), self._local(n)
        p = A.vector(self._device())
        pl = p.getLocalView()
        if self._has_pre:
            self.precond(b, r)
            normb = self.norm(r)
        else:
            normb = self.norm(b)
        if normb == 0.0:
            normb = 1.0
        A.vectorProduct(x, r)
        axpby(1.0, b, -1.0, r)  # r = b - A x
        if self._has_pre:
            self.precond(r, z)
            pl.copy_(z)
            s1 = self.dot(r, z)
        else:
            pl.copy_(r)
            s1 = self.dot(r, r)
        self.iterations = 0
        self.residue = np.sqrt(s1) / normb
        while self.next_iteration():
            A.vectorProduct(p, Ap)
            s2 = self.dot(Ap, pl)
            if s2 == 0.0:
                self.residue = 0.0
                break
            alpha = s1 / s2
            axpby(alpha, pl, 1.0, xl)
            axpby(-alpha, Ap, 1.0, r)
            s2 = s1
            if self._has_pre:
                self.precond(r, z)
                s1 = self.dot(r, z)
            else:
                s1 = self.dot(r, r)
            beta = 0.0 if s2 == 0.0 else s1 / s2
            axpby(1.0, z if self._has_pre else r, beta, pl)
            self.residue = np.sqrt(s1) / normb
        return self.converged()


class BICGStab(_DistSolver):
    """Solvers::Linear::BICGStab over a DistributedMatrix (BICGStab.hpp:33-145)."""

    def __init__(self, matrix, exact_residue=False, **kw):
        super().__init__(matrix, **kw)
        self.exact = bool(exact_residue)

    def _residual(self, x, b, out, tmp):
        from . import axpby
        # out = M^-1 (b - A x)
        if self._has_pre:
            self.A.vectorProduct(x, tmp)
            axpby(1.0, b, -1.0, tmp)
            self.precond(tmp, out)
        else:
            self.A.vectorProduct(x, out)
            axpby(1.0, b, -1.0, out)

    def solve(self, b, x: DistributedVector) -> bool:
        from . import axpby
        A = self.A
        n = A.plan.n_local
        xl = x.getLocalView()
        r, r_ast, Ap, As, tmp, sres = (self._local(n) for _ in range(6))
        p, s = A.vector(self._device()), A.vector(self._device())
        pl, sl = p.getLocalView(), s.getLocalView()
        if self._has_pre:
            self.precond(b, tmp)
            b_norm = self.norm(tmp)
        else:
            b_norm = self.norm(b)
        if b_norm == 0.0:
            b_norm = 1.0
        self._residual(x, b, r, tmp)
        pl.copy_(r)
        r_ast.copy_(r)
        rho = self.dot(r, r_ast)
        r_ast_sqnorm = rho
        eps2 = np.finfo(np.float64 if A.real == "double" else np.float32).eps ** 2
        self.iterations = 0
        self.residue = np.sqrt(rho) / b_norm
        while self.next_iteration():
            # Ap = M^-1 A p ; alpha = rho / (Ap, r_ast)
            if self._has_pre:
                A.vectorProduct(p, tmp)
                self.precond(tmp, Ap)
            else:
                A.vectorProduct(p, Ap)
            alpha = rho / self.dot(Ap, r_ast)
            # s = r - alpha Ap
            sl.copy_(r)
            axpby(-alpha, Ap, 1.0, sl)
            # As = M^-1 A s ; omega = (As, s) / (As, As)
            if self._has_pre:
                A.vectorProduct(s, tmp)
                self.precond(tmp, As)
            else:
                A.vectorProduct(s, As)
            omega = self.dot(As, sl) / self.dot(As, As)
            # x += alpha p + omega s ; r = s - omega As
            axpby(alpha, pl, 1.0, xl)
            axpby(omega, sl, 1.0, xl)
            r.copy_(sl)
            axpby(-omega, As, 1.0, r)
            rho_old = rho
            rho = self.dot(r, r_ast)
            if abs(rho) < eps2 * r_ast_sqnorm:
                # r has become too orthogonal to r_ast: restart with a new r0
                self._residual(x, b, r, tmp)
                r_ast.copy_(r)
                rho = r_ast_sqnorm = self.dot(r, r_ast)
            beta = (rho / rho_old) * (alpha / omega)
            # p = r + beta p - beta omega Ap
            axpby(1.0, r, beta, pl)
            axpby(-beta * omega, Ap, 1.0, pl)
            if self.exact:
                self._residual(x, b, sres, tmp)
                self.residue = self.norm(sres) / b_norm
            else:
                self.residue = self.norm(r) / b_norm
        return self.converged()


class TFQMR(_DistSolver):
    """Solvers::Linear::TFQMR over a DistributedMatrix (TFQMR.hpp:18-114)."""

    def solve(self, b, x: DistributedVector) -> bool:
        from . import axpby
        A = self.A
        n = A.plan.n_local
        xl = x.getLocalView()
        d, r, w, v, r_ast, Au, tmp = (self._local(n) for _ in range(7))
        u = A.vector(self._device())
        ul = u.getLocalView()

        def pmatvec(src, dst):
            if self._has_pre:
                A.vectorProduct(src, tmp)
                self.precond(tmp, dst)
            else:
                A.vectorProduct(src, dst)

        if self._has_pre:
            self.precond(b, tmp)
            b_norm = self.norm(tmp)
            A.vectorProduct(x, tmp)
            axpby(1.0, b, -1.0, tmp)
            self.precond(tmp, r)
        else:
            b_norm = self.norm(b)
            A.vectorProduct(x, r)
            axpby(1.0, b, -1.0, r)
        w.copy_(r)
        ul.copy_(r)
        pmatvec(u, Au)
        v.copy_(Au)
        tau = self.norm(r)
        theta = eta = 0.0
        r_ast.copy_(r)
        rho = self.dot(r_ast, r)
        alpha = 0.0
        if b_norm == 0.0:
            b_norm = 1.0
        self.iterations = 0
        self.residue = tau / b_norm
        while self.next_iteration():
            it = self.iterations
            if it % 2 == 1:
                alpha = rho / self.dot(v, r_ast)
            else:
                pmatvec(u, Au)
            axpby(-alpha, Au, 1.0, w)
            axpby(1.0, ul, theta * theta * eta / alpha, d)
            theta = self.norm(w) / tau
            c = 1.0 / np.sqrt(1.0 + theta * theta)
            tau = tau * theta * c
            eta = c * c * alpha
            axpby(eta, d, 1.0, xl)
            self.residue = tau * np.sqrt(it + 1) / b_norm
            if it > self.minit and self.residue < self.tol:
                break
            if it % 2 == 0:
                rho_new = self.dot(w, r_ast)
                beta = rho_new / rho
                rho = rho_new
                axpby(1.0, w, beta, ul)
                axpby(beta, Au, beta * beta, v)
                pmatvec(u, Au)
                axpby(1.0, Au, 1.0, v)
            else:
                axpby(-alpha, v, 1.0, ul)
        return self.converged()


class GMRES(_DistSolver):
    """Solvers::Linear::GMRES over a DistributedMatrix (GMRES.hpp:76-176 for the
    restart loop with Baker-Jessup-Kolev adaptivity of the restart length,
    192-338 for classical / modified Gram-Schmidt, with reorthogonalisation in
    the R variants, 641-700 for the update, 720-760 for the Givens rotations).

    Every basis vector is a DistributedVector, so the product A v_i
    synchronises its ghosts in place. Each (w, v_k) of modified Gram-Schmidt
    is one all-reduce, as TNL's distributed scalar product; classical
    Gram-Schmidt reduces its i + 1 local projections in ONE all-reduce of the
    coefficient vector (TNL's multireduction over the local rows, GMRES.hpp:
    211-213, sums no other rank's part). The Hessenberg matrix, the rotations
    and the back substitution are host scalars in FP64, identical on every rank
    because every rank sees the same reduced values. The compact-WY variant is
    not provided here (single-GPU GMRES provides it)."""

    VARIANTS = ("CGS", "CGSR", "MGS", "MGSR")

    def __init__(self, matrix, variant="MGSR", restarting_min=10, restarting_max=10, restarting_step_min=3,
                 restarting_step_max=3, **kw):
        if variant not in self.VARIANTS:
            raise ValueError(f"distributed GMRES variants: {', '.join(self.VARIANTS)}")
        super().__init__(matrix, **kw)
        self.variant = variant
        self.rmin, self.rmax = int(restarting_min), int(restarting_max)
        self.dmin, self.dmax = int(restarting_step_min), int(restarting_step_max)

    def _pmatvec(self, v: DistributedVector, dst, tmp):
        # dst = M^-1 A v
        if self._has_pre:
            self.A.vectorProduct(v, tmp)
            self.precond(tmp, dst)
        else:
            self.A.vectorProduct(v, dst)

    def _residual(self, x, b, r, tmp):
        from . import axpby
        # r = M^-1 (b - A x)
        if self._has_pre:
            self.A.vectorProduct(x, tmp)
            axpby(1.0, b, -1.0, tmp)
            self.precond(tmp, r)
        else:
            self.A.vectorProduct(x, r)
            axpby(1.0, b, -1.0, r)

    def _projections(self, V, i, w):
        """The i + 1 coefficients (w, v_k), local dots on the device, one all-reduce."""
        from . import dot
        acc = self._coef
        for k in range(i + 1):
            dot(V[k].getLocalView(), w, acc[k:k + 1])
        self.g.allreduce_sum(acc[:i + 1])
        return acc[:i + 1].tolist()

    @staticmethod
    def _rotation(dx, dy):
        # generatePlaneRotation (GMRES.hpp:720-738)
        if dy == 0.0:
            return 1.0, 0.0
        if abs(dy) > abs(dx):
            t = dx / dy
            sn = 1.0 / np.sqrt(1.0 + t * t)
            return t * sn, sn
        t = dy / dx
        cs = 1.0 / np.sqrt(1.0 + t * t)
        return cs, t * cs

    @staticmethod
    def _rotate(dx, dy, cs, sn):
        # applyPlaneRotation (GMRES.hpp:740-748)
        return cs * dx + sn * dy, cs * dy - sn * dx

    def _cycle(self, m, normb, beta, V, r, w, tmp):
        """One restart cycle of at most m steps; returns (k, H, s) with k the
        index of the last basis vector to use in the update and whether all m
        steps ran."""
        from . import axpby
        H = np.zeros((m + 1, m))
        s = np.zeros(m + 1)
        cs, sn = np.zeros(m + 1), np.zeros(m + 1)
        s[0] = beta
        axpby(1.0 / beta, r, 0.0, V[0].getLocalView())  # v_0 = r / |r|
        cgs = self.variant in ("CGS", "CGSR")
        passes = 2 if self.variant in ("CGSR", "MGSR") else 1
        for i in range(m):
            if not self.next_iteration():
                # not reached: the check before it saw the same state
                return i - 1, H, s, False
            self._pmatvec(V[i], w, tmp)
            for _ in range(passes):
                if cgs:
                    h = self._projections(V, i, w)
                    for k in range(i + 1):
                        H[k, i] += h[k]
                        axpby(-h[k], V[k].getLocalView(), 1.0, w)
                else:
                    for k in range(i + 1):
                        hk = self.dot(w, V[k].getLocalView())
                        H[k, i] += hk
                        axpby(-hk, V[k].getLocalView(), 1.0, w)
            normw = self.norm(w)
            H[i + 1, i] = normw
            axpby(1.0 / normw, w, 0.0, V[i + 1].getLocalView())
            # apply_givens_rotations (GMRES.hpp:750-760)
            for k in range(i):
                H[k, i], H[k + 1, i] = self._rotate(H[k, i], H[k + 1, i], cs[k], sn[k])
            if H[i + 1, i] != 0.0:
                cs[i], sn[i] = self._rotation(H[i, i], H[i + 1, i])
                H[i, i], H[i + 1, i] = self._rotate(H[i, i], H[i + 1, i], cs[i], sn[i])
                s[i], s[i + 1] = self._rotate(s[i], s[i + 1], cs[i], sn[i])
            self.residue = abs(s[i + 1]) / normb
            if not self.check_next():
                return i, H, s, False
        return m - 1, H, s, True

    @staticmethod
    def _update(k, H, s, V, xl):
        """Back substitution H[:k+1, :k+1] y = s[:k+1], then x += V y (GMRES.hpp:641-700)."""
        from . import axpby
        y = s.copy()
        for i in range(k, -1, -1):
            if H[i, i] == 0.0:
                raise ZeroDivisionError("GMRES: singular Hessenberg matrix in the update")
            y[i] /= H[i, i]
            for j in range(i - 1, -1, -1):
                y[j] -= H[j, i] * y[i]
        for j in range(k + 1):
            axpby(y[j], V[j].getLocalView(), 1.0, xl)

    def solve(self, b, x: DistributedVector) -> bool:
        import torch
        if self.rmin <= 0 or self.rmax <= 0 or self.rmin > self.rmax:
            raise ValueError(f"GMRES restarting parameters: r_min = {self.rmin}, r_max = {self.rmax}")
        if self.dmin < 0 or self.dmax < 0 or self.dmin > self.dmax:
            raise ValueError(f"GMRES restarting steps: d_min = {self.dmin}, d_max = {self.dmax}")
        A = self.A
        n = A.plan.n_local
        xl = x.getLocalView()
        r, w, tmp = (self._local(n) for _ in range(3))
        V = [A.vector(self._device()) for _ in range(self.rmax + 1)]
        self._coef = torch.zeros(self.rmax + 1, dtype=torch.float64, device=self._device())
        if self._has_pre:
            self.precond(b, tmp)
            normb = self.norm(tmp)
        else:
            normb = self.norm(b)
        if normb == 0.0:
            normb = 1.0
        self._residual(x, b, r, tmp)
        beta = self.norm(r)
        self.iterations = 0
        self.residue = beta / normb
        beta_ratio, cycles, m = 1.0, 0, self.rmax
        while self.check_next():
            # restart length (Baker, Jessup, Kolev 2009), GMRES.hpp:120-140
            if self.rmax > self.rmin and cycles > 0:
                if beta_ratio > 0.99:
                    m = self.rmax
                elif beta_ratio >= 0.175:
                    step = int(self.dmin + np.float32(self.dmax - self.dmin) / (self.rmax - self.rmin) * (m - self.rmin))
                    m = m - step if m - step >= self.rmin else self.rmax
            k, H, s, full = self._cycle(m, normb, beta, V, r, w, tmp)
            if not full:
                self._update(k, H, s, V, xl)
                return self.converged()
            self._update(m - 1, H, s, V, xl)
            self._residual(x, b, r, tmp)
            beta_old, beta = beta, self.norm(r)
            self.residue = beta / normb
            cycles += 1
            beta_ratio = beta / beta_old
        return self.converged()
