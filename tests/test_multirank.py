"""The multi-rank path of bench.py (one replica per rank, max-over-ranks
timing, whole-job throughput) with world_size 2 on the gloo backend, CPU only."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r measured (1 + r) ms per step and (10 - r) ms end to end
        ms, e2e = bench.max_over_ranks(torch, dist, [1.0 + rank, 10.0 - rank], "cpu")
        out[rank] = (ms, e2e, bench.job_throughput(1e9, ms, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_gloo():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    assert set(res) == {0, 1}
    for r in range(world):
        ms, e2e, gbs = res[r]
        assert ms == 2.0 and e2e == 10.0           # the slowest rank sets the step time
        assert gbs == pytest.approx(2 * 1e9 / 2e-3 / 1e9)  # both replicas' bytes


def test_reference_arm_is_rank_zero_only(monkeypatch, capsys):
    """Under torchrun only rank 0 runs the reference (CPU) arm."""
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class A:
        steps, warmup = 1, 3
    bench.run_reference(A())
    assert capsys.readouterr().out == ""
