"""The request server (continuous batching of solves, include/b2s.h "Serving").

* every result is the same alone and in the mix: each request is solved once
  on a server with one slot (alone) and once among all the others on a
  server with four slots; the solutions must agree to 1e-12 relative
  (max |x_mix - x_alone| / max |x_alone|) — the kernels are deterministic,
  so in practice they agree bit for bit;
* each mixed-precision result reaches the FP64 tolerance 1e-10 on the true
  residual ||b - A x|| / ||b||, and agrees with TNL's own FP64 host solve
  (the oracle) to 1e-7 relative on small cases;
* admission keeps the reserved device memory within the budget and fails a
  request larger than the whole budget with B2S_BUDGET;
* a request asking for mixed precision below the server's mixed_min_rows runs
  the plain FP64 solver (the result says so) and meets the same tolerance; the
  other tests set mixed_min_rows = -1 so that their small requests do run in
  mixed precision.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from b2s import workloads as W
    reqs = []
    reqs.append(("poisson2d", W.poisson2d(40, 31), "cg"))
    reqs.append(("poisson2d", W.poisson2d(150), "cg"))
    reqs.append(("diffusion3d", W.diffusion3d(14, seed=5), "cg"))
    reqs.append(("diffusion3d", W.diffusion3d(24, seed=6), "cg"))
    reqs.append(("convdiff3d", W.convdiff3d(12, seed=7), "bicgstab"))
    reqs.append(("convdiff3d", W.convdiff3d(20, seed=8), "gmres"))
    reqs.append(("convdiff3d", W.convdiff3d(16, seed=9), "bicgstab"))
    reqs.append(("poisson2d", W.poisson2d(64, 100), "cg"))
    return reqs


def _run(b2s, reqs, inflight, mixed=True, budget=None, mixed_min_rows=-1):
    from b2s import workloads as W
    srv = b2s.Server(memory_budget=budget, max_inflight=inflight, mixed_min_rows=mixed_min_rows)
    xs, tickets = [], []
    for i, (_, csr, solver) in enumerate(reqs):
        n = len(csr[0]) - 1
        b = W.uniform(n, 100 + i)
        x = np.zeros(n)
        opts = b2s.solve_opts(solver, tol=1e-10, mixed=mixed)
        tickets.append(srv.submit(csr, b, x, opts))
        xs.append((b, x))
    results = [srv.wait(t, timeout=300) for t in tickets]
    stats = srv.stats()
    srv.close()
    return xs, results, stats


def test_same_result_alone_and_in_the_mix(b2s_lib, cuda):
    reqs = _requests()
    alone_x, alone_r, _ = _run(b2s_lib, reqs, inflight=1)
    mix_x, mix_r, stats = _run(b2s_lib, reqs, inflight=4)
    assert stats["peak_inflight"] >= 2, "requests did not overlap"
    for (name, csr, solver), (_, xa), (_, xm), ra, rm in zip(reqs, alone_x, mix_x, alone_r, mix_r):
        assert ra["ok"] and rm["ok"], (name, solver, ra, rm)
        assert ra["true_residual"] <= 1e-10 and rm["true_residual"] <= 1e-10, (name, solver)
        err = np.max(np.abs(xm - xa)) / np.max(np.abs(xa))
        assert err <= 1e-12, (name, solver, err)
        assert ra["iterations"] == rm["iterations"]


def test_server_matches_fp64_oracle(b2s_lib, cuda, oracle):
    from b2s import workloads as W
    reqs = [r for r in _requests() if len(r[1][0]) - 1 <= 5000]
    xs, res, _ = _run(b2s_lib, reqs, inflight=3)
    for (name, csr, solver), (b, x), r in zip(reqs, xs, res):
        assert r["ok"], (name, r)
        kind = {"cg": "cg", "bicgstab": "bicgstab", "gmres": "gmres"}[solver]
        ref = oracle.solve(kind, csr, b, rtol=1e-12)
        err = np.max(np.abs(x - ref["x"])) / np.max(np.abs(ref["x"]))
        assert err <= 1e-7, (name, solver, err)


def test_admission_respects_the_budget(b2s_lib, cuda):
    from b2s import workloads as W
    reqs = _requests()
    # estimate of the largest request, read back from a first run
    _, res, _ = _run(b2s_lib, reqs[:4], inflight=1)
    biggest = max(r["device_bytes"] for r in res)
    budget = int(biggest * 1.6)
    xs, res, stats = _run(b2s_lib, reqs, inflight=4, budget=budget)
    assert all(r["ok"] for r in res)
    assert stats["peak_reserved_bytes"] <= budget
    assert stats["memory_budget"] == budget
    # larger than the whole budget: refused at once
    srv = b2s_lib.Server(memory_budget=budget, max_inflight=2)
    big = W.diffusion3d(60, seed=1)
    n = len(big[0]) - 1
    t = srv.submit(big, np.ones(n), np.zeros(n), b2s_lib.solve_opts("cg", tol=1e-8))
    r = srv.wait(t, timeout=60)
    srv.close()
    assert r["status"] == b2s_lib.BUDGET


def test_latency_timestamps_are_ordered(b2s_lib, cuda):
    _, res, _ = _run(b2s_lib, _requests()[:5], inflight=2)
    for r in res:
        assert r["t_submit_ns"] <= r["t_admit_ns"] <= r["t_done_ns"]
        assert r["device_ms"] > 0


def test_small_mixed_requests_run_in_fp64(b2s_lib, cuda):
    reqs = _requests()[:4]
    nmax = max(len(r[1][0]) - 1 for r in reqs)
    xs_r, routed, _ = _run(b2s_lib, reqs, inflight=2, mixed_min_rows=nmax + 1)
    xs_m, kept, _ = _run(b2s_lib, reqs, inflight=2, mixed_min_rows=-1)
    xs_p, plain, _ = _run(b2s_lib, reqs, inflight=2, mixed=False)
    for (name, csr, solver), (_, xr), (_, xp), r, k, pl in zip(reqs, xs_r, xs_p, routed, kept, plain):
        assert r["ok"] and k["ok"], name
        assert r["precision"] == "fp64" and k["precision"] == "mixed" and pl["precision"] == "fp64"
        assert r["true_residual"] <= 1e-10 and r["refinements"] == 0
        # routed requests are exactly the plain FP64 solves
        assert np.array_equal(xr, xp) and r["iterations"] == pl["iterations"], name
