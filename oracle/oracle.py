"""TEST INFRASTRUCTURE ONLY — the checker, never the product.

ctypes front end for the two CPU checkers of the sparse path:

* ``Oracle``    — our C restatement (``oracle/liboracle.so``, b2s_oracle.c)
* ``Reference`` — TNL's own Devices::Host code compiled from the reference
                  headers (``oracle/_ref/libtnlref.so``, tnlref_driver.cpp)

Both expose the same calls: ``convert`` (storage arrays of a format, as TNL
lays them out), ``spmv`` and ``solve``. Only tests/, ``__graft_entry__.smoke``
and the reference legs of bench.py (the CPU baseline, the --impl reference
arm, TNL's host runs beside the library's) may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

FORMATS = {"csr": 0, "ellpack": 1, "slicedellpack": 2, "chunkedellpack": 3, "biellpack": 4,
           "slicedellpack8": 5, "slicedellpack16": 6, "slicedellpack64": 7}
ORG = {"col": 0, "row": 1}
SOLVERS = {"cg": 0, "bicgstab": 1, "gmres": 2, "tfqmr": 3, "bicgstabl": 4}
GMRES_VARIANTS = {"CGS": 0, "CGSR": 1, "MGS": 2, "MGSR": 3}

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build_oracle(tnl_src=None) -> None:
    """Compile liboracle.so, and _ref/libtnlref.so when a TNL source tree is
    given (argument or the TNL_SRC environment variable) and exists."""
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    tnl = tnl_src or os.environ.get("TNL_SRC")
    if tnl and Path(tnl).is_dir():
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"TNL_SRC={tnl}"], check=True)


class _Lib:
    prefix = ""
    path: Path

    def __init__(self):
        if not self.path.exists():
            raise FileNotFoundError(f"{self.path} is not built (run oracle/Makefile)")
        lib = C.CDLL(str(self.path))
        p = self.prefix
        f = getattr(lib, p + "create")
        f.restype = C.c_void_p
        f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p]
        getattr(lib, p + "destroy").argtypes = [C.c_void_p]
        f = getattr(lib, p + "storage_size")
        f.restype = C.c_longlong
        f.argtypes = [C.c_void_p]
        getattr(lib, p + "export_values").argtypes = [C.c_void_p, _f64p]
        getattr(lib, p + "export_columns").argtypes = [C.c_void_p, _i32p]
        f = getattr(lib, p + "meta_count")
        f.restype = C.c_int
        f.argtypes = [C.c_void_p]
        f = getattr(lib, p + "meta_name")
        f.restype = C.c_char_p
        f.argtypes = [C.c_void_p, C.c_int]
        f = getattr(lib, p + "meta_size")
        f.restype = C.c_longlong
        f.argtypes = [C.c_void_p, C.c_int]
        getattr(lib, p + "meta_get").argtypes = [C.c_void_p, C.c_int, _i64p]
        f = getattr(lib, p + "spmv")
        f.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int]
        for name in ("permute_rows", "permute_columns"):
            f = getattr(lib, p + name)
            f.restype = C.c_int
            f.argtypes = [C.c_void_p, _i32p]
        f = getattr(lib, p + "reorder")
        f.restype = C.c_void_p
        f.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _i32p, _i32p]
        f = getattr(lib, p + "from_coo")
        f.restype = C.c_void_p
        f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong, _i32p, _i32p, _f64p, C.c_int,
                      C.c_void_p]
        self.lib = lib

    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    # -- matrices ---------------------------------------------------------
    def create(self, fmt: str, org: str, csr, real: str = "f64"):
        off, col, val, ncols = csr
        off = np.ascontiguousarray(off, dtype=np.int32)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        h = self._fn("create")(FORMATS[fmt], ORG[org], {"f64": 0, "f32": 1, "bool": 2}[real],
                               len(off) - 1, int(ncols), off, col, val)
        if not h:
            raise RuntimeError(f"{type(self).__name__}: cannot build {fmt}")
        return h

    def destroy(self, h):
        self._fn("destroy")(h)

    def arrays(self, h) -> dict:
        """Storage arrays (values, columnIndexes) and layout metadata."""
        st = self._fn("storage_size")(h)
        out = {}
        vals = np.empty(max(st, 0), dtype=np.float64)
        cols = np.empty(max(st, 0), dtype=np.int32)
        if st > 0:
            self._fn("export_values")(h, vals)
            self._fn("export_columns")(h, cols)
        out["values"] = vals
        out["columnIndexes"] = cols
        for i in range(self._fn("meta_count")(h)):
            name = self._fn("meta_name")(h, i).decode()
            n = self._fn("meta_size")(h, i)
            a = np.empty(max(n, 1), dtype=np.int64)
            if n > 0:
                self._fn("meta_get")(h, i, a)
            out[name] = a[:n]
        return out

    def convert(self, fmt: str, org: str, csr, real: str = "f64") -> dict:
        h = self.create(fmt, org, csr, real)
        try:
            return self.arrays(h)
        finally:
            self.destroy(h)

    # -- permutations (Matrices/MatrixPermutationApplier.h, SparseOperations.h) --
    def permute_rows(self, csr, perm) -> dict:
        """permuteMatrixRows on a CSR matrix: the arrays of the result."""
        h = self.create("csr", "col", csr)
        try:
            if self._fn("permute_rows")(h, np.ascontiguousarray(perm, dtype=np.int32)) != 0:
                raise RuntimeError("permute_rows failed")
            return self.arrays(h)
        finally:
            self.destroy(h)

    def permute_columns(self, fmt: str, org: str, csr, iperm) -> dict:
        """permuteMatrixColumns on the matrix in layout `fmt`: the arrays of the result."""
        h = self.create(fmt, org, csr)
        try:
            if self._fn("permute_columns")(h, np.ascontiguousarray(iperm, dtype=np.int32)) != 0:
                raise RuntimeError("permute_columns failed")
            return self.arrays(h)
        finally:
            self.destroy(h)

    def reorder(self, csr, perm, iperm) -> dict:
        """reorderSparseMatrix( A, B, perm, iperm ) into a CSR matrix: its arrays."""
        off, col, val, ncols = csr
        h = self._fn("reorder")(len(off) - 1, int(ncols), np.ascontiguousarray(off, dtype=np.int32),
                                np.ascontiguousarray(col, dtype=np.int32), np.ascontiguousarray(val, dtype=np.float64),
                                np.ascontiguousarray(perm, dtype=np.int32), np.ascontiguousarray(iperm, dtype=np.int32))
        if not h:
            raise RuntimeError("reorder failed")
        try:
            return self.arrays(h)
        finally:
            self.destroy(h)

    # -- assembly (SparseMatrixView.hpp:256-340) ----------------------------
    def from_coo(self, fmt: str, org: str, rows, cols, ri, ci, v, add=False, real="f64", caps=None,
                 save_to=None) -> dict:
        """setRowCapacities( caps or the per-row counts ) + setElement /
        addElement per triplet: the arrays (and, for the reference, the matrix
        saved to `save_to` with SparseMatrix::save)."""
        ri = np.ascontiguousarray(ri, dtype=np.int32)
        ci = np.ascontiguousarray(ci, dtype=np.int32)
        v = np.ascontiguousarray(v, dtype=np.float64)
        caps = None if caps is None else np.ascontiguousarray(caps, dtype=np.int32)
        h = self._fn("from_coo")(FORMATS[fmt], ORG[org], 0 if real == "f64" else 1, int(rows), int(cols), len(ri),
                                 ri, ci, v, int(bool(add)), None if caps is None else caps.ctypes.data)
        if not h:
            raise RuntimeError(f"{type(self).__name__}: from_coo failed")
        try:
            if save_to is not None and self.lib.tnlref_save(h, str(save_to).encode()) != 0:
                raise RuntimeError("save failed")
            return self.arrays(h)
        finally:
            self.destroy(h)

    def spmv(self, fmt: str, org: str, csr, x, y=None, alpha=1.0, beta=0.0, begin=0, end=0, real="f64"):
        h = self.create(fmt, org, csr, real)
        try:
            nrows = len(csr[0]) - 1
            yy = np.zeros(nrows) if y is None else np.array(y, dtype=np.float64, copy=True)
            self._fn("spmv")(h, np.ascontiguousarray(x, dtype=np.float64), yy, alpha, beta, begin, end)
            return yy
        finally:
            self.destroy(h)


class Oracle(_Lib):
    """Our C restatement of TNL's algorithms (b2s_oracle.c)."""
    prefix = "b2so_"
    path = HERE / "liboracle.so"

    # how the reference build evaluates ILU(0) (g++ -O3 -march=x86-64-v3): the
    # factorization updates as fused multiply-adds in both precisions; the FP64
    # substitution sums uncontracted; the FP32 sums vectorized by four (products
    # rounded, subtracted in order) with a fused scalar remainder
    ILU_FUSED = {"f64": 1 | 8, "f32": 1 | 8 | 16}

    def __init__(self):
        super().__init__()
        f = self.lib.b2so_ilu0_apply
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        f = self.lib.b2so_solve
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double,
                      C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                      C.POINTER(C.c_longlong), C.POINTER(C.c_double)]

    def spmv_symmetric(self, csr, x, y0=None, alpha=1.0, beta=0.0, begin=0, end=0):
        """SymmetricMatrix product: csr holds the lower triangle."""
        off, col, val, _ = csr
        n = len(off) - 1
        y = np.zeros(n) if y0 is None else np.array(y0, dtype=np.float64, copy=True)
        f = self.lib.b2so_spmv_symmetric
        f.restype = None
        f.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int]
        f(n, np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
          np.ascontiguousarray(val, np.float64), np.ascontiguousarray(x, np.float64), y, alpha, beta, begin, end)
        return y

    def ilu0_apply(self, csr, b, real="f64"):
        """Preconditioners::ILU0 update + solve: x = U^-1 L^-1 b."""
        off, col, val, _ = csr
        n = len(off) - 1
        x = np.zeros(n)
        if self.lib.b2so_ilu0_apply(0 if real == "f64" else 1, self.ILU_FUSED[real], n,
                                    np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
                                    np.ascontiguousarray(val, np.float64), np.ascontiguousarray(b, np.float64), x) != 0:
            raise RuntimeError("ILU(0): a diagonal entry is missing")
        return x

    def solve(self, solver, csr, b, x0=None, rtol=1e-8, maxit=10**9, precond=False,
              gmres_variant="MGSR", restart_min=30, restart_max=30, exact_residue=False, ell=1):
        off, col, val, _ = csr
        n = len(off) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        it = C.c_longlong(0)
        res = C.c_double(0)
        ok = self.lib.b2so_solve(SOLVERS[solver], int(precond), n,
                                 np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
                                 np.ascontiguousarray(val, np.float64), np.ascontiguousarray(b, np.float64),
                                 x, rtol, maxit, GMRES_VARIANTS[gmres_variant], restart_min, restart_max,
                                 int(exact_residue), int(ell), C.byref(it), C.byref(res))
        return {"x": x, "converged": bool(ok), "iterations": it.value, "residue": res.value}


class Reference(_Lib):
    """TNL's own Devices::Host implementation (compiled from the reference headers)."""
    prefix = "tnlref_"
    path = HERE / "_ref" / "libtnlref.so"

    def __init__(self):
        super().__init__()
        lib = self.lib
        lib.tnlref_set_threads.argtypes = [C.c_int]
        lib.tnlref_get_threads.restype = C.c_int
        lib.tnlref_spmv_time.restype = C.c_double
        lib.tnlref_spmv_time.argtypes = [C.c_void_p, _f64p, C.c_int]
        lib.tnlref_read_mtx.restype = C.c_void_p
        lib.tnlref_read_mtx.argtypes = [C.c_int, C.c_int, C.c_int, C.c_char_p]
        lib.tnlref_save.restype = C.c_int
        lib.tnlref_save.argtypes = [C.c_void_p, C.c_char_p]
        lib.tnlref_load.restype = C.c_void_p
        lib.tnlref_load.argtypes = [C.c_int, C.c_int, C.c_int, C.c_char_p]
        lib.tnlref_convert.restype = C.c_void_p
        lib.tnlref_convert.argtypes = [C.c_void_p, C.c_int, C.c_int]
        lib.tnlref_write_mtx.restype = C.c_int
        lib.tnlref_write_mtx.argtypes = [C.c_void_p, C.c_char_p]
        f = lib.tnlref_solve
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double,
                      C.c_longlong, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                      C.POINTER(C.c_longlong), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        f = lib.tnlref_solve_stationary
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_longlong,
                      C.c_double, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
        lib.tnlref_ilut_create.restype = C.c_void_p
        lib.tnlref_ilut_create.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_double]
        lib.tnlref_ilut_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        lib.tnlref_ilut_factors.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _i32p, _i32p, _f64p]
        lib.tnlref_ilut_solve.argtypes = [C.c_void_p, _f64p, _f64p]
        lib.tnlref_ilut_destroy.argtypes = [C.c_void_p]
        lib.tnlref_set_ilut.argtypes = [C.c_int, C.c_double]
        lib.tnlref_mdiag_create.restype = C.c_void_p
        lib.tnlref_mdiag_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f64p]
        lib.tnlref_mdiag_storage.restype = C.c_longlong
        lib.tnlref_mdiag_storage.argtypes = [C.c_void_p]
        lib.tnlref_mdiag_values.argtypes = [C.c_void_p, _f64p]
        lib.tnlref_mdiag_spmv.argtypes = [C.c_void_p, _f64p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int]
        lib.tnlref_mdiag_destroy.argtypes = [C.c_void_p]

    def read_mtx(self, fmt: str, org: str, path, real="f64"):
        """MatrixReader::readMtx into a matrix of layout `fmt`: its arrays, or
        None when TNL's reader throws."""
        h = self.lib.tnlref_read_mtx(FORMATS[fmt], ORG[org], 0 if real == "f64" else 1, str(path).encode())
        if not h:
            return None
        try:
            return self.arrays(h)
        finally:
            self.destroy(h)

    def assign_to(self, fmt: str, org: str, csr, to_fmt: str, to_org: str = "col", real="f64") -> dict:
        """The matrix built from `csr` in layout `fmt`, assigned by operator= to
        layout `to_fmt`: the arrays of the result."""
        h = self.create(fmt, org, csr, real)
        try:
            h2 = self.lib.tnlref_convert(h, FORMATS[to_fmt], ORG[to_org])
            if not h2:
                raise RuntimeError("operator= failed")
            try:
                return self.arrays(h2)
            finally:
                self.destroy(h2)
        finally:
            self.destroy(h)

    def save(self, fmt: str, org: str, csr, path, real="f64"):
        """SparseMatrix::save( fileName ) of the matrix built from `csr` in layout `fmt`."""
        h = self.create(fmt, org, csr, real)
        try:
            if self.lib.tnlref_save(h, str(path).encode()) != 0:
                raise RuntimeError("save failed")
        finally:
            self.destroy(h)

    def load(self, fmt: str, org: str, path, real="f64"):
        """SparseMatrix::load( fileName ) into layout `fmt`: the arrays, or None when TNL throws."""
        h = self.lib.tnlref_load(FORMATS[fmt], ORG[org], 0 if real == "f64" else 1, str(path).encode())
        if not h:
            return None
        try:
            return self.arrays(h)
        finally:
            self.destroy(h)

    def write_mtx(self, fmt: str, org: str, csr, path, real="f64"):
        """MatrixWriter::writeMtx of the matrix built from `csr` in layout `fmt`."""
        h = self.create(fmt, org, csr, real)
        try:
            if self.lib.tnlref_write_mtx(h, str(path).encode()) != 0:
                raise RuntimeError("writeMtx failed")
        finally:
            self.destroy(h)

    def export_range(self, h, name: str, first: int, count: int) -> np.ndarray:
        """Elements [first, first + count) of "values" (as float64) or
        "columnIndexes" (int32) of a matrix made by ``create``."""
        f = self.lib.tnlref_export_range
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_longlong, C.c_void_p]
        out = np.empty(count, dtype=np.float64 if name == "values" else np.int32)
        if f(h, 0 if name == "values" else 1, first, count, out.ctypes.data) != 0:
            raise ValueError("range outside the storage")
        return out

    def meta(self, h) -> dict:
        """The layout's index arrays and scalars (int64), without the storage arrays."""
        out = {}
        for i in range(self._fn("meta_count")(h)):
            name = self._fn("meta_name")(h, i).decode()
            n = self._fn("meta_size")(h, i)
            a = np.empty(max(n, 1), dtype=np.int64)
            if n > 0:
                self._fn("meta_get")(h, i, a)
            out[name] = a[:n]
        return out

    def binary_spmv_f32(self, h, x, y, alpha=1.0, beta=0.0, begin=0, end=0):
        """vectorProduct of a binary matrix (real="bool" in create) with float
        vectors; y (float32) is updated in place."""
        f = self.lib.tnlref_binary_spmv_f32
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS"),
                      np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS"), C.c_double, C.c_double,
                      C.c_int, C.c_int]
        if f(h, np.ascontiguousarray(x, np.float32), y, alpha, beta, begin, end) != 0:
            raise RuntimeError("reference raised")
        return y

    def set_threads(self, n: int):
        self.lib.tnlref_set_threads(int(n))

    def threads(self) -> int:
        return self.lib.tnlref_get_threads()

    def ilu0_apply(self, csr, b, real="f64"):
        """TNL's Preconditioners::ILU0 update + solve: x = U^-1 L^-1 b."""
        off, col, val, _ = csr
        n = len(off) - 1
        x = np.zeros(n)
        f = self.lib.tnlref_ilu0_apply
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        if f(0 if real == "f64" else 1, n, np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
             np.ascontiguousarray(val, np.float64), np.ascontiguousarray(b, np.float64), x) != 0:
            raise RuntimeError("TNL's ILU0 raised")
        return x

    def spmv_time(self, h, x, loops: int) -> float:
        return self.lib.tnlref_spmv_time(h, np.ascontiguousarray(x, dtype=np.float64), loops)

    def spmv_symmetric(self, csr, x, y0=None, alpha=1.0, beta=0.0, begin=0, end=0, real="f64"):
        """SparseMatrix< Real, Host, int, SymmetricMatrix, CSR >::vectorProduct;
        csr holds the lower triangle."""
        off, col, val, _ = csr
        n = len(off) - 1
        y = np.zeros(n) if y0 is None else np.array(y0, dtype=np.float64, copy=True)
        f = self.lib.tnlref_spmv_symmetric
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_double, C.c_double, C.c_int, C.c_int]
        if f(0 if real == "f64" else 1, n, np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
             np.ascontiguousarray(val, np.float64), np.ascontiguousarray(x, np.float64), y, alpha, beta, begin,
             end) != 0:
            raise RuntimeError("reference raised")
        return y

    def solve_stationary(self, solver, csr, b, x0=None, rtol=1e-8, maxit=10**9, omega=1.0, period=4, real="f64"):
        """Solvers::Linear::Jacobi ("jacobi") or SOR ("sor"); SOR's sweep is
        TNL's sequential one with one OpenMP thread (set_threads(1))."""
        off, col, val, _ = csr
        n = len(off) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        it = C.c_longlong(0)
        res = C.c_double(0)
        ok = self.lib.tnlref_solve_stationary({"jacobi": 5, "sor": 6}[solver], 0 if real == "f64" else 1, n,
                                              np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
                                              np.ascontiguousarray(val, np.float64), np.ascontiguousarray(b, np.float64),
                                              x, rtol, maxit, omega, period, C.byref(it), C.byref(res))
        if ok < 0:
            raise RuntimeError("reference solver raised")
        return {"x": x, "converged": bool(ok), "iterations": it.value, "residue": res.value}

    def ilut(self, csr, p=0, tau=1e-4, real="f64"):
        """Preconditioners::ILUT::update( A ): the factors as TNL stores them
        (L: unit diagonal implied; U: rows in reverse order, diagonal first;
        both CSR with their capacity slots, column -1 where unused) and a
        handle for ``ilut_solve``; release it with ``ilut_destroy``."""
        off, col, val, _ = csr
        n = len(off) - 1
        h = self.lib.tnlref_ilut_create(0 if real == "f64" else 1, n, np.ascontiguousarray(off, np.int32),
                                        np.ascontiguousarray(col, np.int32), np.ascontiguousarray(val, np.float64),
                                        int(p), float(tau))
        if not h:
            raise RuntimeError("reference ILUT raised")
        nl, nu = C.c_longlong(0), C.c_longlong(0)
        self.lib.tnlref_ilut_sizes(h, C.byref(nl), C.byref(nu))
        F = {"Loff": np.zeros(n + 1, np.int32), "Lcol": np.zeros(max(nl.value, 1), np.int32),
             "Lval": np.zeros(max(nl.value, 1)), "Uoff": np.zeros(n + 1, np.int32),
             "Ucol": np.zeros(max(nu.value, 1), np.int32), "Uval": np.zeros(max(nu.value, 1))}
        self.lib.tnlref_ilut_factors(h, F["Loff"], F["Lcol"], F["Lval"], F["Uoff"], F["Ucol"], F["Uval"])
        for k, m in (("L", nl.value), ("U", nu.value)):
            F[k + "col"], F[k + "val"] = F[k + "col"][:m], F[k + "val"][:m]
        return h, F

    def multidiagonal(self, rows, cols, offsets, values, real="f64", org="col"):
        """MultidiagonalMatrix( rows, cols, offsets ) with setElement of
        values[r, d] (a rows x len(offsets) array) wherever the column is inside
        the matrix; returns a handle for mdiag_values / mdiag_spmv."""
        offsets = np.ascontiguousarray(offsets, np.int32)
        vals = np.ascontiguousarray(values, np.float64).reshape(-1)
        h = self.lib.tnlref_mdiag_create(0 if real == "f64" else 1, 1 if org == "col" else 0, rows, cols,
                                         len(offsets), offsets, vals)
        if not h:
            raise RuntimeError("reference MultidiagonalMatrix raised")
        return h

    def mdiag_values(self, h):
        out = np.zeros(max(self.lib.tnlref_mdiag_storage(h), 1))
        self.lib.tnlref_mdiag_values(h, out)
        return out[:self.lib.tnlref_mdiag_storage(h)]

    def mdiag_spmv(self, h, x, y0, alpha=1.0, beta=0.0, begin=0, end=0):
        y = np.array(y0, dtype=np.float64, copy=True)
        self.lib.tnlref_mdiag_spmv(h, np.ascontiguousarray(x, np.float64), y, alpha, beta, begin, end)
        return y

    def mdiag_destroy(self, h):
        self.lib.tnlref_mdiag_destroy(h)

    def ilut_solve(self, h, b):
        x = np.zeros(len(b))
        self.lib.tnlref_ilut_solve(h, np.ascontiguousarray(b, np.float64), x)
        return x

    def ilut_destroy(self, h):
        self.lib.tnlref_ilut_destroy(h)

    def solve(self, solver, csr, b, x0=None, rtol=1e-8, maxit=10**9, precond=False,
              gmres_variant="MGSR", restart_min=30, restart_max=30, exact_residue=False, real="f64", ell=1):
        off, col, val, _ = csr
        n = len(off) - 1
        x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        it = C.c_longlong(0)
        res = C.c_double(0)
        sec = C.c_double(0)
        ok = self.lib.tnlref_solve(SOLVERS[solver], int(precond), 0 if real == "f64" else 1, n,
                                   np.ascontiguousarray(off, np.int32), np.ascontiguousarray(col, np.int32),
                                   np.ascontiguousarray(val, np.float64), np.ascontiguousarray(b, np.float64),
                                   x, rtol, maxit, gmres_variant.encode(), restart_min, restart_max,
                                   int(exact_residue), int(ell), C.byref(it), C.byref(res), C.byref(sec))
        if ok < 0:
            raise RuntimeError("reference solver raised")
        return {"x": x, "converged": bool(ok), "iterations": it.value, "residue": res.value,
                "seconds": sec.value}

