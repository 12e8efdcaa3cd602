"""Generate the golden fixtures of tests/golden from TNL itself.

Runs TNL's own Devices::Host code (oracle/_ref/libtnlref.so, compiled from the
reference headers by oracle/Makefile) on seeded matrices and stores:

* layouts.npz  — storage arrays of every segment layout (values, columnIndexes
                 and the layout metadata), ColumnMajorOrder (TNL's Devices::Cuda
                 organization) for FP64 and FP32, RowMajorOrder for FP64
* spmv.npz     — y = A x for a seeded x, per matrix, layout and value type
* solvers.npz  — CG / BiCGStab / GMRES / TFQMR / BiCGStab(ell) results (x, iterations, residue,
                 converged) at rtol 1e-10

Usage (where the reference tree is available):  python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT / "oracle"), str(ROOT / "tnl-dev_b200"), str(ROOT / "tests")]

from oracle import Reference, build_oracle  # noqa: E402
from b2s import workloads as W  # noqa: E402 - numpy-only module
import tnl_unit_matrices as U  # noqa: E402

FORMATS = ["csr", "ellpack", "slicedellpack", "chunkedellpack", "biellpack",
           "slicedellpack8", "slicedellpack16", "slicedellpack64"]


def with_zeros_and_empty_rows():
    off, col, val, nc = W.irregular(400, seed=8, hi=100)
    val = val.copy()
    val[::7] = 0.0  # explicit zeros: dropped by the padded layouts
    lens = np.diff(off)
    lens[[0, 5, 6, 7, 100, 399]] = 0  # empty rows
    keep = np.concatenate([np.arange(off[r], off[r] + lens[r]) for r in range(400)])
    noff = np.zeros(401, dtype=np.int32)
    noff[1:] = np.cumsum(lens)
    return noff, col[keep], val[keep], nc


def matrices():
    return {
        "poisson16": W.poisson2d(16),
        "poisson_7x5": W.poisson2d(7, 5),
        "laplace6": W.laplace3d(6),
        "irregular_zeros_empty": with_zeros_and_empty_rows(),
        "irregular_long": W.irregular(120, seed=7, mu=np.log(40.0), sigma=1.5, hi=1200, ncols=2000),
        "irregular_33": W.irregular(33, seed=9, hi=60),
        "long_rows_129": U.long_rows(129)[0],
        "triangular_90": U.large_triangular(90)[0],
        "convdiff5": W.convdiff3d(5),
        "one_by_one": (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0]), 1),
    }


def main():
    build_oracle()
    R = Reference()
    R.set_threads(1)
    mats = matrices()
    layouts, spmv, solvers, csrs = {}, {}, {}, {}
    for name, csr in mats.items():
        off, col, val, nc = csr
        csrs[f"{name}/offsets"] = off
        csrs[f"{name}/columns"] = col
        csrs[f"{name}/values"] = val
        csrs[f"{name}/ncols"] = np.array([nc])
        x = W.uniform(nc, 1)
        for fmt in FORMATS:
            for org, real in (("col", "f64"), ("col", "f32"), ("row", "f64")):
                arrs = R.convert(fmt, org, csr, real)
                if fmt == "biellpack":
                    # TNL sizes BiEllpack storage as 32 * groupPointers[last] but addresses
                    # only the first groupPointers[last] slots; the rest stays padding.
                    used = int(arrs["groupPointers"][-1])
                    assert np.all(arrs["columnIndexes"][used:] == -1) and np.all(arrs["values"][used:] == 0)
                    arrs["values"] = arrs["values"][:used]
                    arrs["columnIndexes"] = arrs["columnIndexes"][:used]
                for k, v in arrs.items():
                    layouts[f"{name}/{fmt}/{org}/{real}/{k}"] = v
            for real in ("f64", "f32"):
                spmv[f"{name}/{fmt}/{real}"] = R.spmv(fmt, "col", csr, x, real=real)
        spmv[f"{name}/x"] = x
    cases = [
        ("poisson16", "cg", False, "MGSR", 30, 30),
        ("poisson16", "cg", True, "MGSR", 30, 30),
        ("poisson16", "bicgstab", False, "MGSR", 30, 30),
        ("poisson16", "gmres", False, "MGSR", 30, 30),
        ("poisson16", "gmres", False, "CGSR", 30, 30),
        ("laplace6", "cg", True, "MGSR", 30, 30),
        ("convdiff5", "bicgstab", False, "MGSR", 30, 30),
        ("convdiff5", "bicgstab", True, "MGSR", 30, 30),
        ("convdiff5", "gmres", False, "MGSR", 10, 30),
        ("convdiff5", "gmres", True, "CGSR", 30, 30),
        ("convdiff5", "gmres", False, "MGS", 30, 30),
        ("poisson16", "tfqmr", False, "MGSR", 30, 30),
        ("poisson16", "tfqmr", True, "MGSR", 30, 30),
        ("convdiff5", "tfqmr", False, "MGSR", 30, 30),
        ("convdiff5", "tfqmr", True, "MGSR", 30, 30),
        # BiCGStab(ell): the solver field carries ell
        ("poisson16", "bicgstabl1", False, "MGSR", 30, 30),
        ("convdiff5", "bicgstabl2", False, "MGSR", 30, 30),
        ("convdiff5", "bicgstabl2", True, "MGSR", 30, 30),
        ("laplace6", "bicgstabl3", True, "MGSR", 30, 30),
        ("convdiff5", "bicgstabl4", False, "MGSR", 30, 30),
    ]
    for mname, solver, pre, var, rmin, rmax in cases:
        csr = mats[mname]
        n = len(csr[0]) - 1
        rows = np.repeat(np.arange(n), np.diff(csr[0]))
        b = np.zeros(n)
        np.add.at(b, rows, csr[2])  # b = A * ones
        ell = int(solver[9:]) if solver.startswith("bicgstabl") else 1
        r = R.solve(solver[:9] if ell > 1 or solver.startswith("bicgstabl") else solver, csr, b, rtol=1e-10,
                    precond=pre, gmres_variant=var, restart_min=rmin, restart_max=rmax, ell=ell)
        key = f"{mname}/{solver}/{int(pre)}/{var}/{rmin}/{rmax}"
        solvers[f"{key}/x"] = r["x"]
        solvers[f"{key}/b"] = b
        solvers[f"{key}/stats"] = np.array([r["iterations"], r["residue"], float(r["converged"])])
    np.savez_compressed(HERE / "matrices.npz", **csrs)
    np.savez_compressed(HERE / "layouts.npz", **layouts)
    np.savez_compressed(HERE / "spmv.npz", **spmv)
    np.savez_compressed(HERE / "solvers.npz", **solvers)
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")))


if __name__ == "__main__":
    main()
