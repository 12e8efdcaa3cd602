"""Access to the golden fixtures produced from TNL itself (tests/golden/make_golden.py)."""
from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
FORMATS = ["csr", "ellpack", "slicedellpack", "chunkedellpack", "biellpack",
           "slicedellpack8", "slicedellpack16", "slicedellpack64"]
SEGMENTS = {"csr": "CSR", "ellpack": "Ellpack", "slicedellpack": "SlicedEllpack",
            "chunkedellpack": "ChunkedEllpack", "biellpack": "BiEllpack",
            "slicedellpack8": "SlicedEllpack", "slicedellpack16": "SlicedEllpack",
            "slicedellpack64": "SlicedEllpack"}
# SlicedEllpack< ..., SliceSize > of each format name (0: the default 32)
SLICE = {"slicedellpack8": 8, "slicedellpack16": 16, "slicedellpack64": 64}


@lru_cache(None)
def _load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def matrix_names():
    return sorted({k.split("/")[0] for k in _load("matrices")})


def csr(name):
    m = _load("matrices")
    return (m[f"{name}/offsets"], m[f"{name}/columns"], m[f"{name}/values"], int(m[f"{name}/ncols"][0]))


def layout(name, fmt, org, real):
    z = _load("layouts")
    pre = f"{name}/{fmt}/{org}/{real}/"
    return {k[len(pre):]: v for k, v in z.items() if k.startswith(pre)}


def spmv(name, fmt, real):
    z = _load("spmv")
    return z[f"{name}/x"], z[f"{name}/{fmt}/{real}"]


def solver_cases():
    z = _load("solvers")
    keys = sorted({k.rsplit("/", 1)[0] for k in z})
    out = []
    for k in keys:
        mname, solver, pre, var, rmin, rmax = k.split("/")
        it, res, conv = z[f"{k}/stats"]
        ell = 1
        if solver.startswith("bicgstabl"):  # BiCGStab(ell): the key's solver field carries ell
            solver, ell = "bicgstabl", int(solver[9:])
        out.append(dict(key=k, matrix=mname, solver=solver, ell=ell, precond=bool(int(pre)), variant=var,
                        restart_min=int(rmin), restart_max=int(rmax), b=z[f"{k}/b"], x=z[f"{k}/x"],
                        iterations=int(it), residue=float(res), converged=bool(conv)))
    return out


def compare_layout(got: dict, want: dict, fmt: str):
    """Assert bit-exact equality of two layout dicts; for BiEllpack only the
    addressed part of the storage is compared and the rest must be padding."""
    assert set(want) <= set(got), f"missing arrays {set(want) - set(got)}"
    for k, w in want.items():
        g = got[k]
        if fmt == "biellpack" and k in ("values", "columnIndexes"):
            used = len(w)
            tail = g[used:]
            assert np.all(tail == (-1 if k == "columnIndexes" else 0)), f"{k}: non-padding in the unaddressed tail"
            g = g[:used]
        assert g.shape == w.shape, f"{k}: shape {g.shape} != {w.shape}"
        if k == "values":
            assert np.array_equal(g.astype(np.float64), w.astype(np.float64)), f"{k} differs"
        else:
            assert np.array_equal(g.astype(np.int64), w.astype(np.int64)), f"{k} differs"
