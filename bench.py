"""Benchmark of the sparse hot path: SpMV HBM throughput on B200.

Workload (one step = one SpMV over one matrix): the 3D 7-point Laplacian on a
128^3 grid (2,097,152 rows, 14,581,760 nonzeros), CSR, FP64 values, int32
indices, x ~ U[-1,1] (seeded) — the headline cell of the SpMV format sweep.
The rest of the sweep (CSR / Ellpack / SlicedEllpack / ChunkedEllpack /
BiEllpack, FP64 and FP32, on the Laplacian and on the seeded irregular
2M-row log-normal matrix) is reported in the same JSON line.

value   = algorithmic bytes / device time of the SpMV kernel (CUDA events on the
          launching stream; before every step, outside the events, a 256 MiB
          write evicts the matrix and vectors from L2 and a 256 MiB read of a
          second buffer then forces the write-back of those dirty lines, so
          the timed kernel pays for its own traffic only)
          B_spmv = nnz*(s_v+s_i) + (n+1)*s_i + n_cols*s_x + n*s_y
e2e     = the same bytes / time of the public call b2s_spmv with host vectors
          (pinned), H2D of x and D2H of y inside the timed region
Multi-GPU (torchrun): independent replicas, one per GPU (weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-sweep]
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for p in (ROOT / "tnl-dev_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

METRIC = "SpMV HBM GB/s"
L2_FLUSH_BYTES = 256 << 20


def spmv_bytes(n, ncols, nnz, sv, si=4):
    return nnz * (sv + si) + (n + 1) * si + ncols * sv + n * sv


def tnl_bytes(nnz, sv, si=4):
    # TNL's own bandwidth figure (src/Benchmarks/SpMV/spmv.h:714)
    return nnz * (2 * sv + si)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch from the committed ncu summary, or None."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed work runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "samples": len(sm),
                "reasons": sorted(reasons)}


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workloads():
    """The seeded matrix generators (numpy only), loaded by file path so that
    the reference arm never imports the b2s package or its CUDA library."""
    mod = sys.modules.get("b2s_workloads")
    if mod is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("b2s_workloads", ROOT / "tnl-dev_b200" / "b2s" / "workloads.py")
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        sys.modules["b2s_workloads"] = mod
    return mod


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def headline_config(n, nnz, B, ws):
    """The workload named in both arms' JSON lines (identical keys and values)."""
    return {"workload": "spmv_csr_f64_laplace3d_128", "matrix": "3D 7-point Laplacian 128^3",
            "rows": n, "nnz": nnz, "format": "CSR", "index": "int32", "bytes_per_step": B,
            "l2": "inputs larger than L2 (217 MB per step); the GPU arm also evicts L2 before every step "
                  "(256 MiB write + 256 MiB read of a second buffer, outside the events)",
            "parallelism": f"replicas x{ws}"}


def make_matrix(name):
    W = workloads()
    if name == "laplace3d_128":
        return W.laplace3d(128)
    if name == "irregular_2m":
        return W.irregular(2_000_000, seed=2)
    raise KeyError(name)


# ---------------------------------------------------------------------------
# Multi-GPU: independent replicas, one per rank; the step time of the job is
# the slowest rank's, the throughput counts every rank's work.
def max_over_ranks(torch, dist, values, device):
    """Element-wise maximum of per-rank timings (all ranks get the result)."""
    t = torch.tensor([float(v) for v in values], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_throughput(bytes_per_step, ms_per_step, world_size):
    """GB/s of the whole job: every replica moves bytes_per_step per step."""
    return world_size * bytes_per_step / (ms_per_step * 1e-3) / 1e9


# ---------------------------------------------------------------------------
class L2Flush:
    """Evict L2 between timed steps: write a buffer larger than L2, then read a
    second one so the flush's own dirty lines are written back before the
    timed kernel starts."""

    def __init__(self, torch):
        self.w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.r = torch.zeros(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        self.sink = torch.empty((), dtype=torch.float32, device="cuda")

    def fill_(self, v):
        self.w.fill_(v)
        torch_sum = self.r.sum()
        self.sink.copy_(torch_sum)


def time_spmv(torch, A, x, y, steps, warmup, flush):
    """Per-step device time of one SpMV (events on the launching stream)."""
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        flush.fill_(1.0)
        A.vectorProduct(x, y, stream=stream)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for s, e in evs:
        flush.fill_(1.0)  # evict the matrix and vectors from L2 between steps
        s.record(stream)
        A.vectorProduct(x, y, stream=stream)
        e.record(stream)
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in evs]


def time_e2e(torch, A, n, ncols, real, steps, warmup):
    """Public API with host vectors: H2D x, SpMV, D2H y per step (pinned buffers)."""
    dt = torch.float64 if real == "double" else torch.float32
    xh = torch.empty(ncols, dtype=dt).pin_memory()
    yh = torch.empty(n, dtype=dt).pin_memory()
    xh.copy_(torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, ncols)).to(dt))
    xn, yn = xh.numpy(), yh.numpy()
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        A.vectorProduct(xn, yn, stream=stream)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(steps):
        A.vectorProduct(xn, yn, stream=stream)
    e.record(stream)
    torch.cuda.synchronize()
    return s.elapsed_time(e) / steps, xh.numel() * xh.element_size(), yh.numel() * yh.element_size()


def run_ours(args):
    import torch
    import b2s
    ws, rank, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    peak, peak_kind = measured_peaks()
    flush = L2Flush(torch)

    csr = make_matrix("laplace3d_128")
    off, col, val, ncols = csr
    n, nnz = len(off) - 1, len(col)
    A = b2s.SparseMatrix.from_csr(off, col, val, ncols, segments="CSR", real="double")
    x = torch.tensor(np.random.default_rng(1).uniform(-1, 1, ncols), device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    B = spmv_bytes(n, ncols, nnz, 8)

    with ClockSampler(local) as clk:
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        times = time_spmv(torch, A, x, y, args.steps, args.warmup, flush)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        ms = sum(times) / len(times)
        step_stats = {"min": round(min(times), 5), "median": round(statistics.median(times), 5),
                      "max": round(max(times), 5)}
        dev_status = b2s.lib.b2s_matrix_device_status(A.handle, None)
        e2e_ms, h2d, d2h = time_e2e(torch, A, n, ncols, "double", args.steps, max(3, args.warmup))
        sweep = run_sweep(torch, b2s, flush, args) if (rank == 0 and args.sweep) else None
        solves = run_solves(torch, b2s, cases_only=args.solve_cases.split(",") if args.solve_cases else None) \
            if (rank == 0 and args.solves) else None
        serving = run_serving(b2s, quick=args.serving_quick) if (rank == 0 and args.serving) else None
        batched = run_batched(torch, b2s, nsys=args.batch_systems, cluster=args.batch_cluster) \
            if (rank == 0 and args.batched) else None
        tnl_cuda = run_tnl_cuda(sweep, solves) if (rank == 0 and args.tnl_cuda) else None
        tuned = run_autotune(b2s) if (rank == 0 and args.autotune) else None
        assembly = run_assembly(torch, b2s) if (rank == 0 and args.assembly) else None
        ilu = run_ilu(torch, b2s) if (rank == 0 and args.ilu) else None
    if dist is not None:
        ms, e2e_ms = max_over_ranks(torch, dist, [ms, e2e_ms], "cuda")
    value = job_throughput(B, ms, ws)
    e2e_value = job_throughput(B, e2e_ms, ws)
    per_launch_gbs = B / (ms * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 5), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 3D Laplacian)",
            "config": headline_config(n, nnz, B, ws),
            "tnl_metric_gbs": round(tnl_bytes(nnz, 8) / (ms * 1e-3) / 1e9, 1),
            "roofline": {"bound": "hbm", "achieved": round(per_launch_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(per_launch_gbs / peak, 4), "peak_kind": peak_kind,
                         "traffic": profile_traffic("csr_group_kernel_laplace3d_128_f64")},
            "e2e": {"value": round(e2e_value, 1), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms, 4)},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "step_ms": step_stats,
            "device_status": "ok" if dev_status == 0 else f"status {dev_status}",
        }
        if args.cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(csr, B)
        if sweep is not None:
            line["sweep"] = sweep
        if solves is not None:
            line["solves"] = solves
        if serving is not None:
            line["serving"] = serving
        if batched is not None:
            line["batched"] = batched
        if tnl_cuda is not None:
            line["tnl_cuda"] = tnl_cuda
        if tuned is not None:
            line["autotune"] = tuned
        if assembly is not None:
            line["assembly"] = assembly
        if ilu is not None:
            line["ilu0"] = ilu
        line["summary"] = make_summary(line)  # last key: the compact record of every section
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


_MAT_ABBR = {"laplace3d_128": "lap128", "irregular_2m": "irr2m"}
_SEG_ABBR = {"CSR": "CSR", "Ellpack": "Ell", "SlicedEllpack": "SEll", "ChunkedEllpack": "ChEll", "BiEllpack": "BiEll",
             "Multidiagonal": "MDiag"}


def make_summary(line):
    """Every section's headline figures in a few hundred bytes, so that the
    end of the output keeps them: [GB/s, fraction of the measured copy peak]
    per sweep cell; mixed-precision speed-up, iterations and error against
    TNL's host solution per solver; the small CG against TNL's host CG;
    batched solves/s; serving p50/p99 per arrival rate."""
    out = {"headline": [line["value"], line["roofline"]["frac"]], "e2e_gbs": line["e2e"]["value"]}
    cb = line.get("cpu_baseline")
    if cb:
        out["cpu_baseline"] = [cb.get("value"), cb.get("cores"), cb.get("cpu_model")]
    sw = line.get("sweep")
    if sw:
        cells = {}
        for k, v in sw.items():
            m, seg, dt = k.split("/")
            key = f"{_MAT_ABBR.get(m, m)}/{_SEG_ABBR.get(seg, seg)}/{dt}"
            cells[key] = [v["gbs"], v["frac"]] if "gbs" in v else "N/A"
        out["sweep_gbs_frac"] = cells
    sol = line.get("solves")
    if sol:
        c1 = sol.get("poisson2d_256/cg/f64")
        if c1:
            th = c1.get("tnl_host") or {}
            out["cg_poisson256"] = {"gpu_ms": c1["ms"], "its": c1["iterations"], "tnl_host_ms": th.get("ms"),
                                    "tnl_its": th.get("iterations"), "err_vs_tnl": c1.get("error_vs_tnl_host")}
        mixed = {}
        for k, v in sol.items():
            if not k.endswith("/mixed"):
                continue
            base = k[: -len("/mixed")]
            f64 = sol.get(base + "/f64", {})
            m, solver = base.split("/")
            mixed[f"{m.replace('diffusion3d_', 'diff').replace('convdiff3d_', 'cd')}/{solver}"] = {
                "x": v.get("speedup_vs_fp64"), **({"x_vs_csr_f64": v["speedup_vs_csr_fp64"]}
                                                  if "speedup_vs_csr_fp64" in v else {}),
                "ms": [f64.get("ms"), v.get("ms")],
                "its": [f64.get("iterations"), v.get("iterations")],
                "hbm_frac": [(f64.get("traffic") or {}).get("frac"), (v.get("traffic") or {}).get("frac")],
                "err_vs_tnl": [_short(f64.get("error_vs_tnl_host")), _short(v.get("error_vs_tnl_host"))]}
        out["mixed_vs_f64"] = mixed
    bt = line.get("batched")
    if bt:
        out["batched"] = {"solves_per_s": bt["solves_per_s"], "ms": bt["ms"], "gbs": bt["algorithmic_gbs"],
                          "err_vs_tnl": _short(bt.get("sample_error_vs_tnl_host"))}
    sv = line.get("serving")
    if sv:
        out["serving"] = {"sizes": sv.get("size_range"), "n": sv.get("requests_per_rate"),
                          "p50_p99_ms_mixed_f64": {
                              k[5:]: [r["mixed"]["p50_ms"], r["mixed"]["p99_ms"], r["fp64"]["p50_ms"],
                                      r["fp64"]["p99_ms"], r["mixed_vs_fp64_solves_per_s"]]
                              for k, r in sv.items() if k.startswith("rate_")}}
    at = line.get("autotune")
    if at:
        out["autotune"] = {_MAT_ABBR.get(k, k): v["best"] for k, v in at.items()}
    tc = line.get("tnl_cuda")
    if tc:
        out["tnl_cuda"] = tc.get("summary", tc)
    return out


def _short(v):
    return None if v is None else float(f"{v:.2e}")


def run_sweep(torch, b2s, flush, args):
    """GB/s of every layout and value type on both sweep matrices (5 timed steps each)."""
    out = {}
    peak, _ = measured_peaks()
    mats = [m for m in ("laplace3d_128", "irregular_2m") if not args.sweep_matrices or m in args.sweep_matrices.split(",")]
    layouts = [s for s in ("CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack", "Multidiagonal")
               if not args.sweep_layouts or s in args.sweep_layouts.split(",")]
    for mname in mats:
        csr = make_matrix(mname)
        off, col, val, ncols = csr
        n, nnz = len(off) - 1, len(col)
        base = b2s.SparseMatrix.from_csr(off, col, val, ncols, segments="CSR", real="double")
        xs = np.random.default_rng(1).uniform(-1, 1, ncols)
        for real, sv in (("double", 8), ("float", 4)):
            dt = torch.float64 if real == "double" else torch.float32
            x = torch.tensor(xs, dtype=dt, device="cuda")
            y = torch.zeros(n, dtype=dt, device="cuda")
            B = spmv_bytes(n, ncols, nnz, sv)
            for seg in layouts:
                key = f"{mname}/{seg}/{'f64' if sv == 8 else 'f32'}"
                try:
                    t0 = time.time()
                    A = base.convert(seg, real)
                    conv_s = time.time() - t0
                except b2s.B2SError as e:
                    out[key] = {"status": "N/A", "why": str(e).split(":")[1].strip()[:80]}
                    continue
                times = time_spmv(torch, A, x, y, 5, 2, flush)
                ms = statistics.median(times)
                # a Multidiagonal product moves its values (no column indices) and x, y
                Bk = A.getStorageSize() * sv + (n + ncols) * sv if seg == "Multidiagonal" else B
                out[key] = {"gbs": round(Bk / (ms * 1e-3) / 1e9, 1), "frac": round(Bk / (ms * 1e-3) / 1e9 / peak, 3),
                            "ms": round(ms, 4), "convert_s": round(conv_s, 3),
                            "storage": A.getStorageSize(), "bytes": int(Bk)}
                del A
                torch.cuda.empty_cache()
        del base
    return out


def _serving_pool(max_n, levels=8):
    """Request matrices of the serving stream: the three types at sizes spread
    log-uniformly over [1e3, max_n] unknowns (one matrix per type and level)."""
    W = workloads()
    ns = np.exp(np.linspace(np.log(1e3), np.log(max_n), levels))
    pool = {}
    for lvl, n in enumerate(ns):
        k2 = max(8, int(round(np.sqrt(n))))
        k3 = max(6, int(round(n ** (1 / 3))))
        pool[(0, lvl)] = (W.poisson2d(k2), "cg")
        pool[(1, lvl)] = (W.diffusion3d(k3, seed=20 + lvl), "cg")
        pool[(2, lvl)] = (W.convdiff3d(k3, seed=40 + lvl), "bicgstab" if lvl % 2 == 0 else "gmres")
    return pool, ns


def run_serving(b2s, quick=False, rates=(50, 500, 2000), nreq=200, seed=7, slots=16):
    """Seeded Poisson arrival streams of solve requests through b2s.Server:
    p50 / p99 latency (arrival -> solution on the host) and solves/s, mixed
    precision (FP32 inner solves, FP64 refinement to 1e-10) against the plain
    FP64 path on the same stream."""
    import time
    W = workloads()
    max_n = 2e5 if quick else 2e6
    pool, ns = _serving_pool(max_n)
    out = {"sizes": f"log-uniform over {len(ns)} levels in [1e3, {max_n:.0e}] unknowns",
           "size_range": [1e3, max_n],
           "types": "2D 5-pt Laplacian (CG), 3D var-coef diffusion (CG), 3D upwind conv-diff (BiCGStab / GMRES(30))",
           "tolerance": 1e-10, "requests_per_rate": nreq, "slots": slots}
    # one warm-up request per type (module load, pool creation, first graphs)
    srv = b2s.Server(max_inflight=2)
    for t in range(3):
        csr, solver = pool[(t, 0)]
        n = len(csr[0]) - 1
        srv.wait(srv.submit(csr, W.uniform(n, 1), np.zeros(n), b2s.solve_opts(solver, tol=1e-10, mixed=True)))
    srv.close()
    for rate in rates:
        g = np.random.default_rng(seed + rate)
        arrivals = np.cumsum(g.exponential(1.0 / rate, nreq))
        lv = np.clip(np.searchsorted(ns, np.exp(g.uniform(np.log(1e3), np.log(max_n), nreq))), 0, len(ns) - 1)
        kinds = g.integers(0, 3, nreq)
        row = {}
        for label, mixed in (("mixed", True), ("fp64", False)):
            srv = b2s.Server(max_inflight=slots)
            t0 = b2s.Server.clock_ns() + 20_000_000
            tickets, arr = [], []
            for i in range(nreq):
                csr, solver = pool[(int(kinds[i]), int(lv[i]))]
                n = len(csr[0]) - 1
                b = W.uniform(n, 1000 + i)
                x = np.zeros(n)
                due = t0 + int(arrivals[i] * 1e9)
                while b2s.Server.clock_ns() < due:
                    time.sleep(max(0.0, (due - b2s.Server.clock_ns()) * 1e-9 - 2e-4))
                arr.append(due)
                tickets.append(srv.submit(csr, b, x, b2s.solve_opts(solver, tol=1e-10, mixed=mixed,
                                                                    gmres_variant="CGSR")))
            res = [srv.wait(t, timeout=600) for t in tickets]
            st = srv.stats()
            srv.close()
            lat = np.array([(r["t_done_ns"] - a) * 1e-6 for r, a in zip(res, arr)])
            span = (max(r["t_done_ns"] for r in res) - arr[0]) * 1e-9
            svc = np.array([(r["t_done_ns"] - r["t_admit_ns"]) * 1e-6 for r in res])
            build = np.array([(r["t_built_ns"] - r["t_admit_ns"]) * 1e-6 for r in res])
            solve_w = np.array([(r["t_solved_ns"] - r["t_built_ns"]) * 1e-6 for r in res])
            dev = np.array([r["device_ms"] for r in res])
            row[label] = {"p50_ms": round(float(np.percentile(lat, 50)), 3),
                          "service_ms_mean": round(float(svc.mean()), 3),
                          "device_ms_mean": round(float(dev.mean()), 3),
                          "build_ms_mean": round(float(build.mean()), 3),
                          "solve_wall_ms_mean": round(float(solve_w.mean()), 3),
                          "p99_ms": round(float(np.percentile(lat, 99)), 3),
                          "solves_per_s": round(nreq / span, 2),
                          "all_converged": all(r["ok"] for r in res),
                          "max_true_residual": float(max(r["true_residual"] for r in res)),
                          "peak_inflight": st["peak_inflight"]}
        row["mixed_vs_fp64_solves_per_s"] = round(row["mixed"]["solves_per_s"] / row["fp64"]["solves_per_s"], 3)
        out[f"rate_{rate}"] = row
    return out


def run_batched(torch, b2s, nsys=4096, cluster=0):
    """The batched workload: `nsys` shifted 2D Laplacians (n_x, n_y ~ U{32..256},
    shift ~ U[0, 0.1]) with 1..8 right-hand sides ~ U[-1, 1], Jacobi-PCG to
    rtol 1e-8 in one persistent launch; the cluster size per system is
    autotuned on the first solve, the second solve is timed."""
    W = workloads()
    off, col, val, rp, nr = W.batched_poisson2d(nsys, seed=5)
    t_off = torch.from_numpy(off).cuda()
    t_col = torch.from_numpy(col).cuda()
    t_val = torch.from_numpy(val).cuda()
    bt = b2s.BatchedCG(t_off, t_col, t_val, rp, nr, tol=1e-8, cluster_size=cluster)
    del t_off, t_col, t_val
    B = torch.from_numpy(np.random.default_rng(9).uniform(-1, 1, bt.vector_length)).cuda()
    X = torch.zeros_like(B)
    bt.solve(B, X)  # autotune + warm-up
    X.zero_()
    ok = bt.solve(B, X)
    r = bt.report
    its, res, sts = bt.results()
    n_s = np.diff(rp)
    nnz_s = np.diff(off.astype(np.int64)[rp])
    it_max = np.maximum.reduceat(its, bt.rhs_off[:-1])
    per_rhs_vec = its * np.repeat(n_s, nr) * 11 * 8
    mat = it_max * (12 * nnz_s + 4 * (n_s + 1) + 8 * n_s)
    algo_bytes = float(per_rhs_vec.sum() + mat.sum())
    sec = r.device_ms * 1e-3
    # a sample of the batch against TNL's own Devices::Host CG with the
    # Diagonal preconditioner (same right-hand sides, rtol 1e-8)
    sample_err, sample_its = None, None
    R = _reference()
    if R is not None:
        Bh, Xh = B.cpu().numpy(), X.cpu().numpy()
        order = np.argsort(np.diff(rp), kind="stable")
        picks = [int(order[i]) for i in np.linspace(0, nsys - 1, 4).astype(int)]
        sample_err, sample_its = 0.0, []
        for sidx in picks:
            csr = W.batch_system(off, col, val, rp, sidx)
            n, k = csr[3], int(nr[sidx])
            blk = slice(int(bt.vec_off[sidx]), int(bt.vec_off[sidx + 1]))
            for j in range(k):
                t = R.solve("cg", csr, np.ascontiguousarray(Bh[blk].reshape(n, k)[:, j]), rtol=1e-8, precond=True)
                xb = Xh[blk].reshape(n, k)[:, j]
                sample_err = max(sample_err, float(np.max(np.abs(xb - t["x"])) / np.max(np.abs(t["x"]))))
                sample_its.append([int(its[int(bt.rhs_off[sidx]) + j]), int(t["iterations"])])
    return {"systems": nsys, "right_hand_sides": int(r.solves), "unknowns": int(rp[-1]), "nnz": int(len(col)),
            "sample_error_vs_tnl_host": sample_err, "sample_iterations_ours_tnl": sample_its,
            "all_converged": bool(ok), "converged": int(r.converged), "ms": round(r.device_ms, 3),
            "solves_per_s": round(r.solves / sec, 1), "iterations_mean": round(float(its.mean()), 1),
            "iterations_max": int(r.max_iterations), "max_residue": float(r.max_residue),
            "cluster_size": int(r.cluster_size), "algorithmic_gbs": round(algo_bytes / sec / 1e9, 1),
            "launches": 1}


def run_autotune(b2s):
    """The layout autotuner on the two sweep matrices (FP64): the chosen
    layout and the time of every candidate (each product timed with L2
    evicted before it, as the sweep times them)."""
    out = {}
    for name in ("laplace3d_128", "irregular_2m"):
        csr = make_matrix(name)
        A = b2s.SparseMatrix.from_csr(*csr[:3], csr[3])
        best, table = b2s.autotune(A, reps=10)
        fmt = lambda e: e["segments"] + (f"/{e['csr_kernel']}" if e["segments"] == "CSR" else "") + (
            ("/groups" if e["csr_row_groups"] else "/windows") if e["csr_kernel"] == "CSRAdaptive" else "") + (
            f"/tpr{e['threads_per_row']}" if e["csr_kernel"] == "CSRVector" else "") + (
            f"/slice{e['slice_size']}" if e["segments"] == "SlicedEllpack" else "")
        out[name] = {"best": fmt(best), "best_us": round(best["spmv_us"], 2), "l2": "evicted before each product",
                     "candidates_us": {fmt(e): (None if e["skipped"] else round(e["spmv_us"], 2)) for e in table}}
        del A
    return out


def run_assembly(torch, b2s, grid=4096):
    """Device assembly (b2s_matrix_from_coo: setRowCapacities + setElement
    for every triplet) of the 2D 5-point Laplacian on a grid x grid mesh —
    TNL's sparse-setup benchmark matrix (16,777,216 rows at grid 4096) —
    from device-resident triplets in row order (the already-sorted path) and
    in a random order (the radix-sorted path), CSR FP64."""
    n = grid * grid
    r = torch.arange(n, device="cuda", dtype=torch.int64)
    i, j = r // grid, r % grid
    cand = torch.stack([r - grid, r - 1, r, r + 1, r + grid], dim=1)
    ok = torch.stack([i > 0, j > 0, torch.ones_like(i, dtype=torch.bool), j < grid - 1, i < grid - 1], dim=1)
    vals = torch.tensor([-1.0, -1.0, 4.0, -1.0, -1.0], device="cuda", dtype=torch.float64).expand(n, 5)
    rows = r.unsqueeze(1).expand(n, 5)[ok].to(torch.int32).contiguous()
    cols = cand[ok].to(torch.int32).contiguous()
    v = vals[ok].contiguous()
    del r, i, j, cand, ok, vals
    count = rows.numel()
    perm = torch.randperm(count, device="cuda", generator=torch.Generator(device="cuda").manual_seed(1))
    shuffled = (rows[perm].contiguous(), cols[perm].contiguous(), v[perm].contiguous())
    del perm
    out = {"matrix": f"2D 5-point Laplacian {grid}^2", "rows": n, "triplets": count,
           "tnl_published_s": {"setElement on GPU": 0.02481, "getRow": 0.02429, "forElements": 0.02211,
                               "note": "TNL tutorial_Matrices.md sparse setup table, 16,777,216 rows, its GPU"}}
    for name, (ri, ci, vv) in (("sorted", (rows, cols, v)), ("shuffled", shuffled)):
        times = []
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            M = b2s.SparseMatrix.from_coo(n, n, ri, ci, vv)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            del M
        best = min(times)
        # triplets read once (4 + 4 + 8 B) and the CSR written once (12 B / nnz + 4 B / row)
        algo = count * 16 + count * 12 + (n + 1) * 4
        out[name] = {"s": round(best, 4), "triplets_per_s": round(count / best, 1),
                     "algorithmic_gbs": round(algo / best / 1e9, 1)}
    del shuffled, rows, cols, v
    torch.cuda.empty_cache()
    return out


def run_ilu(torch, b2s):
    """ILU(0) (Preconditioners::ILU0) on the 128^3 upwind convection-diffusion
    matrix: factorization and one application M^-1 b on the device, TNL's own
    Devices::Host update + solve on the host cores beside it, and BiCGStab to
    rtol 1e-10 with and without it."""
    W = workloads()
    csr = W.convdiff3d(128, seed=4)
    n = len(csr[0]) - 1
    out = {"matrix": "3D upwind convection-diffusion 128^3", "rows": n}
    M = b2s.SparseMatrix.from_csr(*csr[:3], csr[3])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    P = b2s.Preconditioner(M, "ilu0")
    torch.cuda.synchronize()
    out["factor_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    b = torch.tensor(W.uniform(n, 11), device="cuda")
    x = torch.empty_like(b)
    for _ in range(2):
        P.solve(b, x)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(10):
        P.solve(b, x)
    e.record()
    torch.cuda.synchronize()
    out["apply_ms"] = round(s.elapsed_time(e) / 10, 3)
    try:
        from oracle import Reference
        R = Reference()
        R.set_threads(_ref_threads())
        t0 = time.perf_counter()
        R.ilu0_apply(csr, b.cpu().numpy())
        out["tnl_host_update_and_solve_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
    except (FileNotFoundError, OSError):
        out["tnl_host_update_and_solve_ms"] = None
    for pre in (None, "ilu0"):
        slv = b2s.BICGStab()
        slv.setMatrix(M)
        slv.setPreconditioner(pre)
        slv.setConvergenceResidue(1e-10)
        times = []
        for _ in range(2):
            xx = torch.zeros(n, dtype=torch.float64, device="cuda")
            ok = slv.solve(b, xx)
            times.append(slv.report.device_ms)
        out[f"bicgstab_{pre or 'none'}"] = {"ok": bool(ok), "iterations": int(slv.getIterations()),
                                           "ms": round(min(times), 2)}
    del P, M
    torch.cuda.empty_cache()
    return out


def run_solves(torch, b2s, quick=False, cases_only=None):
    """Krylov solves on the GPU: plain FP64 vs mixed precision (FP32 inner
    solves, FP64 refinement) to a true relative residual of 1e-10, plus the
    small Poisson CG of the plain method (rtol 1e-8).

    Each entry: device ms per solve (CUDA events around the solve), solves/s,
    iterations, true FP64 residual, and for mixed runs the max relative
    difference to the FP64 solution."""
    W = workloads()
    out = {}

    def solve(kind, A, b, mixed, tol, variant="CGSR", precond=False, reps=2):
        ell = int(kind[9:]) if kind.startswith("bicgstabl") else 1
        s = {"cg": b2s.CG, "bicgstab": b2s.BICGStab, "gmres": b2s.GMRES, "tfqmr": b2s.TFQMR,
             "bicgstabl": b2s.BICGStabL}[kind[:9] if kind.startswith("bicgstabl") else kind]()
        s.setMatrix(A)
        s.setConvergenceResidue(tol)
        s.setPreconditioner("diagonal" if precond else None)
        s.setup({"gmres-variant": variant, "gmres-restarting-min": 30, "gmres-restarting-max": 30,
                 "bicgstab-ell": ell})
        s.setPrecision(mixed)
        times = []
        x = None
        for _ in range(reps):
            x = torch.zeros(A.getRows(), dtype=torch.float64, device="cuda")
            ok = s.solve(b, x)
            times.append(s.report.device_ms)
        r = s.report
        return x, {"ok": bool(ok), "ms": round(min(times), 3), "solves_per_s": round(1000.0 / min(times), 3),
                   "iterations": int(r.iterations), "refinements": int(r.refinements),
                   "true_residual": float(r.true_residual)}

    # the plain method's small case: 2D Poisson 256^2, CG, b = A*1, rtol 1e-8
    R = _reference()
    want = (lambda key: cases_only is None or key in cases_only)
    if want("poisson2d_256/cg"):
        _poisson_cg(torch, b2s, W, R, solve, out)
    cases = [("diffusion3d_160" if not quick else "diffusion3d_64", "cg", False)]
    cases += [("convdiff3d_128" if not quick else "convdiff3d_48", k, False)
              for k in ("bicgstab", "gmres", "tfqmr", "bicgstabl2")]
    # the same systems stored as TNL's MultidiagonalMatrix (values only, no column indices)
    cases += [(m + "-mdiag", k, False) for m, k, _ in cases if k in ("cg", "bicgstab", "gmres")]
    cases = [c for c in cases if want(f"{c[0]}/{c[1]}")]
    _mixed_cases(torch, b2s, W, R, solve, out, cases)
    return out


def _poisson_cg(torch, b2s, W, R, solve, out):
    csr = W.poisson2d(256)
    A = b2s.SparseMatrix.from_csr(*csr[:3], csr[3])
    ones = torch.ones(A.getRows(), dtype=torch.float64, device="cuda")
    b = torch.empty_like(ones)
    A.vectorProduct(ones, b)
    x, res = solve("cg", A, b, False, 1e-8, reps=3)
    res["max_error_vs_ones"] = float((x - 1).abs().max())
    # TNL's own CG on the host cores (Devices::Host, OpenMP), the same system
    if R is not None:
        t = R.solve("cg", csr, b.cpu().numpy(), rtol=1e-8)
        res["tnl_host"] = {"ms": round(t["seconds"] * 1e3, 2), "iterations": int(t["iterations"]),
                           "threads": _ref_threads()}
        res["error_vs_tnl_host"] = _rel_err(x, t["x"])
    else:
        res["tnl_host"] = None
    out["poisson2d_256/cg/f64"] = res


def solve_traffic(kind, n, nnz, iterations, refinements, mixed, restart=30, mdiag_storage=None):
    """Algorithmic bytes of a solve (per-iteration formulas of the Krylov loops
    over CSR with int32 indices): CG B_spmv + 9 n s_x; BiCGStab 2 B_spmv +
    15 n s_x; GMRES(m) with re-orthogonalised classical Gram-Schmidt B_spmv +
    (4 (i+1) + 5) n s_x at step i, averaged over a cycle. Mixed precision: the
    inner terms with s_v = s_x = 4, plus per refinement one FP64 product and
    3 n 8 bytes for r = b - A x and x += d. A Multidiagonal matrix
    (mdiag_storage slots) moves mdiag_storage s values and no indices per
    product. None for other solvers."""
    sv = 4 if mixed else 8

    def spmv(s):
        if mdiag_storage is not None:
            return mdiag_storage * s + 2 * n * s
        return nnz * (s + 4) + (n + 1) * 4 + 2 * n * s
    if kind == "cg":
        per = spmv(sv) + 9 * n * sv
    elif kind == "bicgstab":
        per = 2 * spmv(sv) + 15 * n * sv
    elif kind == "gmres":
        per = spmv(sv) + (4 * (restart + 1) / 2 + 5) * n * sv
    else:
        return None
    total = iterations * per
    if mixed:
        total += refinements * (spmv(8) + 3 * n * 8)
    return total


def _mixed_cases(torch, b2s, W, R, solve, out, cases):
    oracle_x = {}
    peak, _ = measured_peaks()
    for mname, kind, pre in cases:
        base, _, layout = mname.partition("-")
        size = int(base.rsplit("_", 1)[1])
        csr = W.diffusion3d(size, seed=3) if mname.startswith("diffusion") else W.convdiff3d(size, seed=4)
        seg = "Multidiagonal" if layout == "mdiag" else "CSR"
        A = b2s.SparseMatrix.from_csr(*csr[:3], csr[3], segments=seg, keep_fp32_copy=True)
        bh = W.uniform(A.getRows(), 11)
        b = torch.tensor(bh, device="cuda")
        # the FP64 oracle solution of this system: TNL's own Devices::Host
        # solver (CG for the SPD matrix, BiCGStab otherwise) to rtol 1e-10
        if R is not None and base not in oracle_x:
            t = R.solve("cg" if mname.startswith("diffusion") else "bicgstab", csr, bh, rtol=1e-10)
            oracle_x[base] = (t["x"], round(t["seconds"] * 1e3, 1), int(t["iterations"]))
        x64, r64 = solve(kind, A, b, False, 1e-10, precond=pre)
        x32, r32 = solve(kind, A, b, True, 1e-10, precond=pre)
        r32["max_rel_diff_vs_fp64"] = float((x32 - x64).abs().max() / x64.abs().max())
        r32["speedup_vs_fp64"] = round(r64["ms"] / r32["ms"], 3)
        n, nnz = A.getRows(), len(csr[1])
        mst = A.getStorageSize() if seg == "Multidiagonal" else None
        for r, mixed in ((r64, False), (r32, True)):
            B = solve_traffic(kind, n, nnz, r["iterations"], r["refinements"], mixed, mdiag_storage=mst)
            if B is not None:
                gbs = B / (r["ms"] * 1e-3) / 1e9
                r["traffic"] = {"bytes_per_iteration": round(B / max(r["iterations"], 1)), "gbs": round(gbs, 1),
                                "frac": round(gbs / peak, 3), "bound_ms": round(B / (peak * 1e9) * 1e3, 3)}
        if seg == "Multidiagonal" and f"{base}/{kind}/f64" in out:
            # the mixed Multidiagonal solve against the plain FP64 solve of the CSR matrix
            r32["speedup_vs_csr_fp64"] = round(out[f"{base}/{kind}/f64"]["ms"] / r32["ms"], 3)
        if base in oracle_x:
            xo, tms, tits = oracle_x[base]
            r64["error_vs_tnl_host"] = _rel_err(x64, xo)
            r32["error_vs_tnl_host"] = _rel_err(x32, xo)
            r64["tnl_host"] = r32["tnl_host"] = {"ms": tms, "iterations": tits, "threads": _ref_threads(),
                                                 "solver": "cg" if mname.startswith("diffusion") else "bicgstab"}
        out[f"{mname}/{kind}/f64"] = r64
        out[f"{mname}/{kind}/mixed"] = r32
        del A
        torch.cuda.empty_cache()


# TNL's own Devices::Cuda SpMV and solvers, compiled from the reference headers
# for sm_100a, were timed beside this library's on the same B200: correct on
# small matrices, but the run over the full-size sweep matrices ended with
# cudaErrorIllegalAddress raised inside TNL (reported by its CUDA allocator,
# Allocators/Cuda.h:81). Reference GPU code that faulted is not run again.
TNL_CUDA_UNAVAILABLE = ("TNL's Devices::Cuda path built for sm_100a raised cudaErrorIllegalAddress (700) on the "
                        "full-size sweep matrices (128^3 Laplacian / 2M irregular) on B200; not run again")


def run_tnl_cuda(sweep, solves):
    """The reference's GPU kernels beside ours: unavailable (see TNL_CUDA_UNAVAILABLE)."""
    return {"unavailable": TNL_CUDA_UNAVAILABLE}


def _reference():
    """TNL's own Devices::Host build (oracle/_ref) with every host thread, or None."""
    try:
        from oracle import Reference
        R = Reference()
    except (FileNotFoundError, OSError):
        return None
    R.set_threads(_ref_threads())
    return R


def _rel_err(x, xref):
    """max_i |x_i - xref_i| / max_i |xref_i| (x a device tensor, xref a host array)."""
    xh = x.double().cpu().numpy()
    return float(np.max(np.abs(xh - xref)) / max(np.max(np.abs(xref)), 1e-300))


def _ref_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(csr, B, budget_s=8.0):
    """TNL's own Devices::Host CSR SpMV (OpenMP, all host threads) on the same matrix."""
    try:
        from oracle import Reference
        R = Reference()
        kind = "reference"
    except (FileNotFoundError, OSError):
        return {"value": None, "unit": "GB/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    threads = _ref_threads()
    R.set_threads(threads)
    h = R.create("csr", "col", csr)
    try:
        x = np.random.default_rng(1).uniform(-1, 1, csr[3])
        t1 = R.spmv_time(h, x, 2)
        loops = max(3, min(200, int(budget_s / max(t1, 1e-4))))
        t = R.spmv_time(h, x, loops)
    finally:
        R.destroy(h)
    return {"value": round(B / t / 1e9, 2), "unit": "GB/s", "cores": threads, "kind": kind, "cpu_model": cpu_model(),
            "sample": f"{loops} CSR SpMVs of the full 128^3 Laplacian (FP64), "
                      f"TNL Devices::Host, {threads} OpenMP threads", "ms_per_spmv": round(t * 1e3, 3)}


def run_reference(args):
    ws, rank, local = dist_info()
    if rank != 0:
        return
    csr = make_matrix("laplace3d_128")
    off, col, val, ncols = csr
    n, nnz = len(off) - 1, len(col)
    B = spmv_bytes(n, ncols, nnz, 8)
    try:
        from oracle import Reference
        R = Reference()
    except (FileNotFoundError, OSError) as e:
        print(json.dumps({"impl": "reference", "unavailable": f"TNL reference build missing: {e}"}))
        return
    threads = _ref_threads()
    R.set_threads(threads)
    h = R.create("csr", "col", csr)
    x = np.random.default_rng(1).uniform(-1, 1, ncols)
    R.spmv_time(h, x, max(1, args.warmup))
    per = [R.spmv_time(h, x, 1) for _ in range(args.steps)]
    R.destroy(h)
    ms = 1e3 * sum(per) / len(per)
    value = B / (ms * 1e-3) / 1e9
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded 3D Laplacian)", "impl": "reference",
            "config": headline_config(n, nnz, B, ws),
            "cpu_baseline": {"value": round(value, 2), "unit": "GB/s", "cores": threads, "kind": "reference",
                             "cpu_model": cpu_model(),
                             "sample": f"one full CSR SpMV per step, TNL Devices::Host, {threads} OpenMP threads"},
            "e2e": {"value": round(value, 2), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-sweep", dest="sweep", action="store_false")
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--no-solves", dest="solves", action="store_false")
    ap.add_argument("--no-serving", dest="serving", action="store_false")
    ap.add_argument("--no-batched", dest="batched", action="store_false")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false")
    ap.add_argument("--no-assembly", dest="assembly", action="store_false")
    ap.add_argument("--no-ilu", dest="ilu", action="store_false")
    ap.add_argument("--no-tnl-cuda", dest="tnl_cuda", action="store_false",
                    help="leave out the record of TNL's own CUDA kernels (unavailable on this GPU)")
    ap.add_argument("--sweep-layouts", default="",
                    help="comma-separated layouts of the sweep (e.g. Multidiagonal); default all")
    ap.add_argument("--sweep-matrices", default="",
                    help="comma-separated sweep matrices (laplace3d_128, irregular_2m); default both")
    ap.add_argument("--solve-cases", default="",
                    help="comma-separated solve cases to run (e.g. diffusion3d_160/cg); default all")
    ap.add_argument("--batch-systems", type=int, default=4096,
                    help="systems of the batched solve (4096: the configured workload; fewer for profiling)")
    ap.add_argument("--batch-cluster", type=int, default=0,
                    help="SMs per system of the batched solve (0: autotuned on the first solve)")
    ap.add_argument("--serving-quick", action="store_true",
                    help="serving stream over sizes 1e3..2e5 only (the default is the full 1e3..2e6 range)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
