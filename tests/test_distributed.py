"""The distributed path's host logic on CPU: TNL's row partition
(Containers/Partitioner.h:30-72), the halo plan (which columns each rank needs
from which owner, the [owned | ghosts] renumbering) and the exchange itself,
with world_size 2 and 3 on the gloo backend and with 4 thread ranks
(LocalGroup), host tensors only. The product of each rank's renumbered rows
with its synchronized [owned | ghosts] vector must equal the same rows of the
global product bit for bit (the rows keep their element order)."""
import os
import socket
import sys
import threading
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _matrix(n=700, seed=5):
    """Random rows with a band plus far entries (every rank needs entries from several others)."""
    sys.path.insert(0, str(ROOT / "tnl-dev_b200"))
    from b2s import workloads as W
    return W.irregular(n, seed=seed, mu=np.log(6), sigma=0.8, hi=60)


def _rowsum(off, col, val, x):
    """Row sums in element order (the same function on both sides of each comparison)."""
    out = np.zeros(len(off) - 1)
    for r in range(len(off) - 1):
        acc = 0.0
        for k in range(off[r], off[r + 1]):
            acc += val[k] * x[col[k]]
        out[r] = acc
    return out


def _check_rank(group, n, csr, x_glob, ranges=None):
    """Build the plan for this rank's rows, exchange, and compare; returns a summary."""
    from b2s.distributed import HaloPlan, DistributedVector, split_range
    off, col, val, _ = csr
    lo, hi = ranges[group.rank] if ranges else split_range(n, group.rank, group.size)
    loff = (off[lo:hi + 1] - off[lo]).astype(np.int32)
    lcol = col[off[lo]:off[hi]]
    lval = val[off[lo]:off[hi]]
    plan = HaloPlan(group, (lo, hi), n, lcol)
    # the ghosts are exactly the off-rank columns referenced, sorted
    want_g = np.unique(lcol[(lcol < lo) | (lcol >= hi)])
    assert np.array_equal(plan.ghosts, want_g)
    v = DistributedVector(group, plan, dtype=torch.float64, device="cpu")
    v.getLocalView().copy_(torch.from_numpy(x_glob[lo:hi]))
    v.synchronize()
    ext = v.getConstLocalViewWithGhosts().numpy()
    assert np.array_equal(ext[hi - lo:], x_glob[plan.ghosts])
    rc = plan.renumber(lcol)
    got = _rowsum(loff, rc, lval, ext)
    want = _rowsum(off, col, val, x_glob)[lo:hi]
    assert np.array_equal(got, want)
    # a second exchange after the owned entries change
    v.getLocalView().mul_(-2.0)
    v.synchronize()
    assert np.array_equal(v.getConstLocalViewWithGhosts().numpy()[hi - lo:], -2.0 * x_glob[plan.ghosts])
    return plan.n_ghosts, sum(len(s) for s in plan.send.values())


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT / "tnl-dev_b200"))
    from datetime import timedelta
    from b2s.distributed import TorchGroup, HaloPlan
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        g = TorchGroup()
        csr = _matrix()
        n = len(csr[0]) - 1
        x = np.random.default_rng(3).uniform(-1, 1, n)
        out[rank] = _check_rank(g, n, csr, x)
        # a bad column on one rank: every rank raises (no rank is left waiting)
        cols = np.array([0, n + 5]) if rank == world - 1 else np.array([0])
        try:
            HaloPlan(g, (0, n) if world == 1 else
                     ((rank * n // world), ((rank + 1) * n // world)), n, cols)
            out[f"bad{rank}"] = "no error"
        except ValueError as e:
            out[f"bad{rank}"] = str(e)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(world):
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    for r in range(world):
        assert r in res
        assert "outside" in res[f"bad{r}"], res[f"bad{r}"]
    # what the ranks receive in total is what they send in total
    assert sum(res[r][0] for r in range(world)) == sum(res[r][1] for r in range(world))
    assert all(res[r][0] > 0 for r in range(world))


def test_halo_exchange_thread_ranks_with_an_empty_rank():
    """Four ranks as threads; rank 2 owns no rows (an uneven split given explicitly)."""
    sys.path.insert(0, str(ROOT / "tnl-dev_b200"))
    from b2s.distributed import LocalGroup
    csr = _matrix(n=400, seed=9)
    n = len(csr[0]) - 1
    ranges = [(0, 150), (150, 260), (260, 260), (260, 400)]
    x = np.random.default_rng(4).uniform(-1, 1, n)
    groups = LocalGroup.world(4, timeout=60)
    res, errs = {}, []

    def run(g):
        try:
            res[g.rank] = _check_rank(g, n, csr, x, ranges)
        except BaseException as e:  # noqa: BLE001 - reported below
            errs.append(e)
            g._w.barrier.abort()

    ts = [threading.Thread(target=run, args=(g,)) for g in groups]
    for t in ts:
        t.start()
    for t in ts:
        t.join(120)
    assert not errs, errs
    assert res[2] == (0, 0)
    assert sum(v[0] for v in res.values()) == sum(v[1] for v in res.values())


def test_partitioner():
    from b2s.distributed import split_range, get_owner, get_offset
    for n in (0, 1, 5, 7, 100, 1001):
        for p in (1, 2, 3, 4, 7, 8):
            rs = [split_range(n, r, p) for r in range(p)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(rs[r][1] == rs[r + 1][0] for r in range(p - 1))
            assert all(get_offset(n, r, p) == min(n, rs[r][0]) or rs[r][0] == n for r in range(p))
            if n:
                i = np.arange(n)
                own = get_owner(i, n, p)
                for r, (a, b) in enumerate(rs):
                    assert np.all(own[a:b] == r)
                if n >= p:  # TNL's own formula (Partitioner.h:44-54) where it is exact
                    tnl = i * p // n
                    bump = (tnl < p - 1) & (i >= np.minimum(tnl + 1, p - 1) * n // p)
                    assert np.array_equal(own, tnl + bump)


def test_bad_ranges_are_refused():
    sys.path.insert(0, str(ROOT / "tnl-dev_b200"))
    from b2s.distributed import LocalGroup, HaloPlan
    groups = LocalGroup.world(2, timeout=30)
    errs = {}

    def run(g, rng):
        try:
            HaloPlan(g, rng, 10, np.array([0, 9]))
        except ValueError as e:
            errs[g.rank] = str(e)

    ts = [threading.Thread(target=run, args=(g, r)) for g, r in zip(groups, [(0, 4), (5, 10)])]
    for t in ts:
        t.start()
    for t in ts:
        t.join(60)
    assert set(errs) == {0, 1} and all("contiguously" in e for e in errs.values())
