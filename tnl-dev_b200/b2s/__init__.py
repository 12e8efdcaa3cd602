"""Python front end of libb2sparse — TNL's sparse hot path on B200.

The classes mirror the TNL interface they replace so that code written
against TNL reads the same:

* ``SparseMatrix``  — ``TNL::Matrices::SparseMatrix< Real, Devices::Cuda, int,
  GeneralMatrix, Segments >`` (Matrices/SparseMatrix.h) with ``vectorProduct``
* ``CG``, ``BICGStab``, ``GMRES`` — ``TNL::Solvers::Linear`` solvers with
  ``setMatrix``, ``setPreconditioner``, ``setConvergenceResidue``,
  ``setMaxIterations``, ``setup``, ``solve( b, x )``, ``getIterations``,
  ``getResidue`` (Solvers/Linear/LinearSolver.h, IterativeSolver.h)

Vectors are torch CUDA tensors (device memory, used in place) or numpy
arrays (host memory, copied in and out by the library). Every call goes
through the C ABI of include/b2s.h; there is no CPU implementation here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import (OK, NOT_CONVERGED, NAN, DIVERGED, OOM, CUDA_ERROR, TIMEOUT, INVALID_ARG, INDEX_OVERFLOW,
                   UNSUPPORTED, BREAKDOWN, BUDGET, CANCELLED, IO_ERROR, F64, F32, BOOL, HOST, DEVICE)

lib = _abi.load()

SEGMENTS = {"CSR": _abi.CSR, "Ellpack": _abi.ELLPACK, "SlicedEllpack": _abi.SLICED_ELLPACK,
            "ChunkedEllpack": _abi.CHUNKED_ELLPACK, "BiEllpack": _abi.BIELLPACK,
            "Multidiagonal": _abi.MULTIDIAGONAL}
# TNL's CSR kernel segment names (Segments/CSR.h:577-605) mapped to ours
CSR_KERNELS = {"CSRDefault": _abi.CSR_AUTO, "CSRScalar": _abi.CSR_SCALAR, "CSRVector": _abi.CSR_VECTOR,
               "CSRLight": _abi.CSR_VECTOR, "CSRHybrid": _abi.CSR_VECTOR, "CSRAdaptive": _abi.CSR_ADAPTIVE}
REALS = {"double": F64, "float": F32, "bool": BOOL, np.float64: F64, np.float32: F32, np.bool_: BOOL}


class B2SError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.b2s_last_error().decode()
        self.status = status
        super().__init__(f"{where}: {lib.b2s_status_string(status).decode()} ({status}) {msg}")


def _matrix_opts(csr_kernel="CSRDefault", threads_per_row=0, keep_fp32_copy=False, slice_size=0,
                 csr_row_groups=True, symmetric=False):
    opts = _abi.MatrixOpts()
    lib.b2s_matrix_opts_default(C.byref(opts))
    opts.csr_kernel = CSR_KERNELS.get(csr_kernel, _abi.CSR_AUTO)
    opts.threads_per_row = threads_per_row
    opts.keep_fp32_copy = int(keep_fp32_copy)
    opts.slice_size = int(slice_size)
    opts.csr_row_groups = 0 if csr_row_groups else -1
    opts.symmetric = int(bool(symmetric))
    return opts


def mtx_read(path):
    """MatrixReader's parsing of a MatrixMarket file (host only, no GPU):
    dict with rows, cols, symmetric and the 0-based triplets in TNL's
    setElement order."""
    p = C.POINTER(_abi.Mtx)()
    check(lib.b2s_mtx_read(str(path).encode(), C.byref(p)), "b2s_mtx_read")
    try:
        m = p.contents
        n = m.count
        out = {"rows": m.rows, "cols": m.cols, "symmetric": bool(m.symmetric),
               "row_indexes": np.ctypeslib.as_array(m.row_indexes, shape=(max(n, 1),))[:n].copy(),
               "column_indexes": np.ctypeslib.as_array(m.column_indexes, shape=(max(n, 1),))[:n].copy(),
               "values": np.ctypeslib.as_array(m.values, shape=(max(n, 1),))[:n].copy()}
    finally:
        lib.b2s_mtx_free(p)
    return out


def check(status: int, where: str):
    if status != OK:
        raise B2SError(status, where)


def _is_torch(v) -> bool:
    return type(v).__module__.startswith("torch")


def _ptr(v, dtype: int):
    """(pointer, where) of a torch CUDA tensor or a numpy array of the right type."""
    if _is_torch(v):
        import torch
        want = torch.float64 if dtype == F64 else torch.float32
        if v.dtype != want or not v.is_contiguous():
            raise TypeError(f"vector must be a contiguous {want} tensor")
        return C.c_void_p(v.data_ptr()), DEVICE if v.is_cuda else HOST
    want = np.float64 if dtype == F64 else np.float32
    if not isinstance(v, np.ndarray) or v.dtype != want or not v.flags.c_contiguous:
        raise TypeError(f"vector must be a contiguous numpy {want.__name__} array")
    return C.c_void_p(v.ctypes.data), HOST


def _stream_ptr(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


class SparseMatrix:
    """TNL::Matrices::SparseMatrix< Real, Devices::Cuda, int, GeneralMatrix, Segments >."""

    def __init__(self, handle, real: int):
        self._h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self.real = real
        info = _abi.MatrixInfo()
        check(lib.b2s_matrix_get_info(self._h, C.byref(info)), "b2s_matrix_get_info")
        self.info = info

    # -- construction -------------------------------------------------------
    @classmethod
    def from_csr(cls, offsets, columns, values, columns_count=None, segments="CSR", real="double",
                 csr_kernel="CSRDefault", threads_per_row=0, keep_fp32_copy=False, slice_size=0, stream=None,
                 csr_row_groups=True, symmetric=False):
        """Assemble from CSR arrays (numpy host arrays or torch CUDA tensors) —
        setRowCapacities + setElement, then operator= into `segments`.
        symmetric=True: SparseMatrix< ..., SymmetricMatrix >, the arrays hold the
        lower triangle (any layout)."""
        fmt = SEGMENTS[segments]
        dt = REALS[real]
        opts = _matrix_opts(csr_kernel, threads_per_row, keep_fp32_copy, slice_size, csr_row_groups, symmetric)
        if _is_torch(offsets):
            import torch
            rows = offsets.numel() - 1
            nnz = columns.numel()
            vdt = F32 if values is not None and values.dtype == torch.float32 else F64
            ptrs = [C.c_void_p(offsets.data_ptr()), C.c_void_p(columns.data_ptr()),
                    C.c_void_p(values.data_ptr()) if values is not None else None]
            where = DEVICE
        else:
            offsets = np.ascontiguousarray(offsets, dtype=np.int32)
            columns = np.ascontiguousarray(columns, dtype=np.int32)
            if values is not None:
                values = np.ascontiguousarray(values)
                if values.dtype not in (np.float64, np.float32):
                    values = values.astype(np.float64)
            rows = len(offsets) - 1
            nnz = len(columns)
            vdt = F32 if values is not None and values.dtype == np.float32 else F64
            ptrs = [C.c_void_p(offsets.ctypes.data), C.c_void_p(columns.ctypes.data),
                    C.c_void_p(values.ctypes.data) if values is not None else None]
            where = HOST
        cols = rows if columns_count is None else int(columns_count)
        h = C.c_void_p()
        check(lib.b2s_matrix_create(fmt, dt, rows, cols, nnz, *ptrs, vdt, where, C.byref(opts),
                                    _stream_ptr(stream), C.byref(h)), "b2s_matrix_create")
        return cls(h, dt)

    @classmethod
    def multidiagonal(cls, rows, columns_count, offsets, values, real="double", keep_fp32_copy=False, stream=None):
        """MultidiagonalMatrix( rows, columns, diagonalsOffsets ) with
        values[r, d] = A(r, r + offsets[d]) (a rows x len(offsets) host array;
        slots whose column lies outside the matrix are ignored). The offsets
        are kept ascending."""
        offsets = np.asarray(offsets, dtype=np.int64)
        order = np.argsort(offsets, kind="stable")
        offsets = offsets[order]
        if len(np.unique(offsets)) != len(offsets):
            raise ValueError("repeated diagonal offset")
        vals = np.asarray(values, dtype=np.float64).reshape(rows, len(offsets))[:, order]
        r = np.repeat(np.arange(rows, dtype=np.int64), len(offsets))
        c = r + np.tile(offsets, rows)
        keep = (c >= 0) & (c < columns_count)
        off = np.concatenate([[0], np.cumsum(keep.reshape(rows, -1).sum(axis=1))]).astype(np.int32)
        return cls.from_csr(off, c[keep].astype(np.int32), vals.reshape(-1)[keep], columns_count,
                            segments="Multidiagonal", real=real, keep_fp32_copy=keep_fp32_copy, stream=stream)

    @classmethod
    def from_coo(cls, rows, columns_count, row_indexes, column_indexes, values, segments="CSR", real="double",
                 duplicates="set", stream=None, csr_kernel="CSRDefault", threads_per_row=0, keep_fp32_copy=False,
                 slice_size=0, csr_row_groups=True, row_capacities=None, symmetric=False):
        """Assemble on the device from triplets (numpy arrays or torch CUDA
        tensors): setRowCapacities( row_capacities, default: per-row triplet
        counts ) + setElement (duplicates="set") or addElement
        (duplicates="add") for every triplet in order. symmetric=True: a
        SymmetricMatrix, (i, j) with i < j is stored at (j, i) (any layout)."""
        opts = _matrix_opts(csr_kernel, threads_per_row, keep_fp32_copy, slice_size, csr_row_groups, symmetric)
        dt = REALS[real]
        if _is_torch(row_indexes):
            import torch
            n = row_indexes.numel()
            vdt = F64 if values.dtype == torch.float64 else F32
            ptrs = [C.c_void_p(t.data_ptr()) for t in (row_indexes, column_indexes, values)]
            where = DEVICE
            caps = None if row_capacities is None else row_capacities.to(torch.int32).contiguous()
            caps_ptr = C.c_void_p(caps.data_ptr()) if caps is not None else None
        else:
            row_indexes = np.ascontiguousarray(row_indexes, dtype=np.int32)
            column_indexes = np.ascontiguousarray(column_indexes, dtype=np.int32)
            values = np.ascontiguousarray(values)
            if values.dtype not in (np.float64, np.float32):
                values = values.astype(np.float64)
            n = len(row_indexes)
            vdt = F64 if values.dtype == np.float64 else F32
            ptrs = [C.c_void_p(a.ctypes.data) for a in (row_indexes, column_indexes, values)]
            where = HOST
            caps = None if row_capacities is None else np.ascontiguousarray(row_capacities, dtype=np.int32)
            caps_ptr = C.c_void_p(caps.ctypes.data) if caps is not None else None
        dup = {"set": _abi.DUP_SET, "add": _abi.DUP_ADD}[duplicates]
        h = C.c_void_p()
        check(lib.b2s_matrix_from_coo(SEGMENTS[segments], dt, int(rows), int(columns_count), n, *ptrs, vdt, where, dup,
                                      caps_ptr, C.byref(opts), _stream_ptr(stream), C.byref(h)),
              "b2s_matrix_from_coo")
        return cls(h, dt)

    @classmethod
    def read_mtx(cls, path, segments="CSR", real="double", stream=None, **kw):
        """MatrixReader::readMtx( fileName, matrix )."""
        opts = _matrix_opts(kw.get("csr_kernel", "CSRDefault"), kw.get("threads_per_row", 0),
                            kw.get("keep_fp32_copy", False), kw.get("slice_size", 0), kw.get("csr_row_groups", True))
        dt = REALS[real]
        h = C.c_void_p()
        check(lib.b2s_matrix_read_mtx(str(path).encode(), SEGMENTS[segments], dt, C.byref(opts), _stream_ptr(stream),
                                      C.byref(h)), "b2s_matrix_read_mtx")
        return cls(h, dt)

    def write_mtx(self, path):
        """MatrixWriter::writeMtx( fileName, matrix )."""
        check(lib.b2s_matrix_write_mtx(self._h, str(path).encode()), "b2s_matrix_write_mtx")

    def save(self, path):
        """SparseMatrix::save( fileName ): TNL's binary format."""
        check(lib.b2s_matrix_save(self._h, str(path).encode()), "b2s_matrix_save")

    @classmethod
    def load(cls, path, slice_size=0, stream=None, **kw):
        """SparseMatrix::load( fileName ): layout and value type from the file."""
        opts = _matrix_opts(kw.get("csr_kernel", "CSRDefault"), kw.get("threads_per_row", 0),
                            kw.get("keep_fp32_copy", False), slice_size, kw.get("csr_row_groups", True))
        h = C.c_void_p()
        check(lib.b2s_matrix_load(str(path).encode(), C.byref(opts), _stream_ptr(stream), C.byref(h)),
              "b2s_matrix_load")
        info = _abi.MatrixInfo()
        check(lib.b2s_matrix_get_info(h, C.byref(info)), "b2s_matrix_get_info")
        return cls(h, info.dtype)

    def convert(self, segments="CSR", real=None, stream=None):
        """operator=( const OtherMatrix& ) into another layout / value type."""
        dt = self.real if real is None else REALS[real]
        h = C.c_void_p()
        check(lib.b2s_matrix_convert(self._h, SEGMENTS[segments], dt, None, _stream_ptr(stream), C.byref(h)),
              "b2s_matrix_convert")
        return SparseMatrix(h, dt)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.b2s_matrix_destroy(h)
            self._h = None

    # -- TNL accessors ------------------------------------------------------
    def getRows(self):
        return self.info.rows

    def getColumns(self):
        return self.info.cols

    def getNonzeroElementsCount(self):
        return self.info.nnz

    def getStorageSize(self):
        return self.info.storage_size

    def isSymmetric(self):
        return bool(self.info.symmetric)

    @property
    def handle(self):
        return self._h

    def export(self, name: str) -> np.ndarray:
        """A storage array in TNL's layout (values, columnIndexes, segment metadata)."""
        cnt = C.c_int64()
        check(lib.b2s_matrix_export(self._h, name.encode(), None, 0, C.byref(cnt)), f"export {name}")
        if name == "values":
            out = np.empty(cnt.value, dtype=np.float64 if self.real == F64 else np.float32)
            if cnt.value == 0:
                return out
        elif name == "columnIndexes":
            out = np.empty(cnt.value, dtype=np.int32)
        else:
            out = np.empty(cnt.value, dtype=np.int64)
        check(lib.b2s_matrix_export(self._h, name.encode(), C.c_void_p(out.ctypes.data), cnt.value, C.byref(cnt)),
              f"export {name}")
        return out

    def export_range(self, name: str, first: int, count: int) -> np.ndarray:
        """Elements [first, first + count) of "values" or "columnIndexes"."""
        dt = (np.float64 if self.real == F64 else np.float32) if name == "values" else np.int32
        out = np.empty(count, dtype=dt)
        check(lib.b2s_matrix_export_range(self._h, name.encode(), int(first), int(count), C.c_void_p(out.ctypes.data)),
              f"export_range {name}")
        return out

    def _refresh(self):
        info = _abi.MatrixInfo()
        check(lib.b2s_matrix_get_info(self._h, C.byref(info)), "b2s_matrix_get_info")
        self.info = info

    @staticmethod
    def _perm(p):
        if _is_torch(p):
            return C.c_void_p(p.data_ptr()), DEVICE, p
        a = np.ascontiguousarray(p, dtype=np.int32)
        return C.c_void_p(a.ctypes.data), HOST, a

    def permuteRows(self, perm, stream=None):
        """Matrices::permuteMatrixRows( *this, perm ): row i becomes the old row perm[i] (CSR)."""
        ptr, where, keep = self._perm(perm)
        check(lib.b2s_matrix_permute_rows(self._h, ptr, where, _stream_ptr(stream)), "b2s_matrix_permute_rows")
        self._refresh()

    def permuteColumns(self, iperm, stream=None):
        """Matrices::permuteMatrixColumns( *this, iperm ): column c becomes iperm[c]."""
        ptr, where, keep = self._perm(iperm)
        check(lib.b2s_matrix_permute_columns(self._h, ptr, where, _stream_ptr(stream)), "b2s_matrix_permute_columns")

    def reorder(self, perm, iperm, stream=None):
        """Matrices::reorderSparseMatrix( *this, B, perm, iperm ): returns B (CSR)."""
        p, where, k1 = self._perm(perm)
        ip, where2, k2 = self._perm(iperm)
        if where != where2:
            raise TypeError("perm and iperm must both be on the host or both on the device")
        h = C.c_void_p()
        check(lib.b2s_matrix_reorder(self._h, p, ip, where, _stream_ptr(stream), C.byref(h)), "b2s_matrix_reorder")
        return SparseMatrix(h, self.real)

    def vectorProduct(self, inVector, outVector, matrixMultiplicator=1.0, outVectorMultiplicator=0.0, begin=0,
                      end=0, stream=None):
        """outVector = matrixMultiplicator * A inVector + outVectorMultiplicator * outVector
        over rows [begin, end) (end == 0: all rows)."""
        vt = self.real
        if vt == BOOL:  # a binary matrix takes FP64 or FP32 vectors (both of one type)
            vt = F32 if str(getattr(inVector, "dtype", "")).endswith("float32") else F64
        px, wx = _ptr(inVector, vt)
        py, wy = _ptr(outVector, vt)
        if wx != wy:
            raise TypeError("in and out vectors must both be on the host or both on the device")
        check(lib.b2s_spmv_ex(self._h, px, py, vt, float(matrixMultiplicator), float(outVectorMultiplicator), begin,
                              end, wx, _stream_ptr(stream)), "b2s_spmv_ex")


# ---------------------------------------------------------------------------
# Preconditioners (Solvers/Linear/Preconditioners): update at construction, solve per use
PRECONDITIONERS = {None: _abi.PRECOND_NONE, "": _abi.PRECOND_NONE, "none": _abi.PRECOND_NONE,
                   "diagonal": _abi.PRECOND_JACOBI, "jacobi": _abi.PRECOND_JACOBI, "ilu0": _abi.PRECOND_ILU0,
                   "ilut": _abi.PRECOND_ILUT}


class Preconditioner:
    """Preconditioners::Diagonal ("diagonal"), ILU0 ("ilu0") or ILUT ("ilut",
    with TNL's "ilut-p" = p and "ilut-threshold" = threshold) of `matrix`:
    update() happens here, solve(b, x) applies M^-1."""

    def __init__(self, matrix: SparseMatrix, kind="ilu0", stream=None, p=0, threshold=1e-4):
        self._h = C.c_void_p()
        self.real = matrix.real
        self.matrix = matrix  # the factors refer to it
        if kind == "ilut":
            check(lib.b2s_precond_create_ilut(matrix.handle, int(p), float(threshold), _stream_ptr(stream),
                                              C.byref(self._h)), "b2s_precond_create_ilut")
            return
        check(lib.b2s_precond_create(matrix.handle, PRECONDITIONERS[kind], _stream_ptr(stream), C.byref(self._h)),
              "b2s_precond_create")

    def solve(self, b, x, stream=None):
        pb, wb = _ptr(b, self.real)
        px, wx = _ptr(x, self.real)
        if wb != wx:
            raise TypeError("b and x must both be on the host or both on the device")
        check(lib.b2s_precond_solve(self._h, pb, px, wb, _stream_ptr(stream)), "b2s_precond_solve")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:
            lib.b2s_precond_destroy(h)
            self._h = None


# ---------------------------------------------------------------------------
# Autotuner of the SpMV layout
FORMAT_NAMES = {v: k for k, v in SEGMENTS.items()}
CSR_KERNEL_NAMES = {_abi.CSR_AUTO: "CSRDefault", _abi.CSR_SCALAR: "CSRScalar", _abi.CSR_VECTOR: "CSRVector",
                    _abi.CSR_ADAPTIVE: "CSRAdaptive"}


def autotune(matrix: SparseMatrix, real=None, reps=10, max_storage_ratio=3.0, stream=None, warm_l2=False):
    """Time vectorProduct of `matrix` (CSR) in every candidate layout; returns
    (best, table): best is a dict of SparseMatrix.from_csr keyword arguments
    plus the measured microseconds, table lists every candidate. Each timed
    product starts with L2 evicted unless warm_l2."""
    dt = matrix.real if real is None else REALS[real]
    o = _abi.TuneOpts()
    lib.b2s_tune_opts_default(C.byref(o))
    o.reps = int(reps)
    o.warm_l2 = int(bool(warm_l2))
    o.max_storage_ratio = float(max_storage_ratio)
    best = _abi.TuneResult()
    cap = 32
    table = (_abi.TuneEntry * cap)()
    cnt = C.c_int32()
    check(lib.b2s_autotune_spmv(matrix.handle, dt, C.byref(o), _stream_ptr(stream), C.byref(best),
                                C.cast(table, C.c_void_p), cap, C.byref(cnt)), "b2s_autotune_spmv")

    def entry(e):
        return {"segments": FORMAT_NAMES[e.format], "csr_kernel": CSR_KERNEL_NAMES.get(e.csr_kernel, "CSRDefault"),
                "threads_per_row": e.threads_per_row, "slice_size": e.slice_size,
                "csr_row_groups": e.csr_row_groups >= 0}

    b = entry(best)
    b["spmv_us"] = best.spmv_us
    rows = []
    for e in table[:min(cnt.value, cap)]:
        d = entry(e)
        d.update({"skipped": bool(e.skipped), "storage_size": e.storage_size, "spmv_us": e.spmv_us})
        rows.append(d)
    return b, rows


# ---------------------------------------------------------------------------
# Algorithms primitives
def _cuda_only(*ts):
    """The device vector ops take CUDA tensors only (a host pointer would reach a kernel)."""
    for t in ts:
        if not (_is_torch(t) and t.is_cuda and t.is_contiguous()):
            raise TypeError("expected contiguous torch CUDA tensors")


def dot(a, b, result, stream=None):
    """result[0] = (a, b) in FP64 on the device (a, b, result torch CUDA tensors)."""
    _cuda_only(a, b, result)
    if a.dtype != b.dtype or a.numel() != b.numel() or str(result.dtype) != "torch.float64":
        raise TypeError("dot: a and b of one type and length, result float64")
    dt = F64 if str(a.dtype) == "torch.float64" else F32
    check(lib.b2s_dot(dt, a.numel(), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                      C.c_void_p(result.data_ptr()), _stream_ptr(stream)), "b2s_dot")


def norm2(a, result, stream=None):
    _cuda_only(a, result)
    if str(result.dtype) != "torch.float64":
        raise TypeError("norm2: result float64")
    dt = F64 if str(a.dtype) == "torch.float64" else F32
    check(lib.b2s_norm2(dt, a.numel(), C.c_void_p(a.data_ptr()), C.c_void_p(result.data_ptr()),
                        _stream_ptr(stream)), "b2s_norm2")


def axpby(alpha, x, beta, y, stream=None):
    _cuda_only(x, y)
    if x.dtype != y.dtype or x.numel() != y.numel():
        raise TypeError("axpby: x and y of one type and length")
    dt = F64 if str(x.dtype) == "torch.float64" else F32
    check(lib.b2s_axpby(dt, x.numel(), float(alpha), C.c_void_p(x.data_ptr()), float(beta),
                        C.c_void_p(y.data_ptr()), _stream_ptr(stream)), "b2s_axpby")


def gather(src, idx, dest, stream=None):
    """dest[i] = src[idx[i]] (torch CUDA tensors; idx int32): the pack step of a halo exchange."""
    _cuda_only(src, idx, dest)
    if str(idx.dtype) != "torch.int32":
        raise TypeError("gather: int32 indices")
    if src.element_size() != dest.element_size() or dest.numel() != idx.numel():
        raise TypeError("gather: dest must have idx's length and src's element type")
    check(lib.b2s_gather(src.element_size(), idx.numel(), C.c_void_p(src.data_ptr()), src.numel(),
                         C.c_void_p(idx.data_ptr()), C.c_void_p(dest.data_ptr()), _stream_ptr(stream)), "b2s_gather")


def reorderArray(src, dest, perm, stream=None):
    """Matrices::reorderArray( src, dest, perm ): dest[i] = src[perm[i]] (torch CUDA tensors)."""
    _cuda_only(src, dest, perm)
    check(lib.b2s_reorder_array(src.element_size(), src.numel(), C.c_void_p(src.data_ptr()),
                                C.c_void_p(dest.data_ptr()), C.c_void_p(perm.data_ptr()), _stream_ptr(stream)),
          "b2s_reorder_array")


def scan_i32(data, inclusive=False, stream=None):
    check(lib.b2s_scan_i32(data.numel(), C.c_void_p(data.data_ptr()), int(inclusive), _stream_ptr(stream)),
          "b2s_scan_i32")


# ---------------------------------------------------------------------------
# Linear solvers
class _LinearSolver:
    kind = _abi.CG

    def __init__(self):
        self.opts = _abi.SolveOpts()
        lib.b2s_solve_opts_default(C.byref(self.opts))
        self.opts.solver = self.kind
        self.matrix = None
        self._solver = None
        self.report = _abi.SolveReport()

    # LinearSolver / IterativeSolver interface
    def setMatrix(self, matrix: SparseMatrix):
        self.matrix = matrix
        self._reset()

    def setPreconditioner(self, name):
        self.opts.preconditioner = PRECONDITIONERS[name]
        self._reset()

    def setConvergenceResidue(self, r):
        self.opts.convergence_residue = float(r)
        self._reset()

    def setDivergenceResidue(self, r):
        self.opts.divergence_residue = float(r)
        self._reset()

    def setMaxIterations(self, n):
        self.opts.max_iterations = int(n)
        self._reset()

    def setMinIterations(self, n):
        self.opts.min_iterations = int(n)
        self._reset()

    def setPrecision(self, mixed: bool, inner_tolerance=None):
        """Mixed precision: FP32 inner solves inside FP64 iterative refinement."""
        self.opts.precision = _abi.PRECISION_MIXED if mixed else _abi.PRECISION_PLAIN
        if inner_tolerance is not None:
            self.opts.inner_tolerance = float(inner_tolerance)
        self._reset()

    def setCheckInterval(self, n):
        self.opts.check_interval = int(n)
        self._reset()

    def setup(self, params: dict, prefix: str = ""):
        """Parameter names of TNL's configuration (ConfigDescription keys)."""
        o = self.opts
        keys = {"convergence-residue": ("convergence_residue", float),
                "divergence-residue": ("divergence_residue", float),
                "max-iterations": ("max_iterations", int), "min-iterations": ("min_iterations", int),
                "gmres-restarting-min": ("gmres_restarting_min", int),
                "gmres-restarting-max": ("gmres_restarting_max", int),
                "gmres-restarting-step-min": ("gmres_restarting_step_min", int),
                "gmres-restarting-step-max": ("gmres_restarting_step_max", int),
                "bicgstab-exact-residue": ("bicgstab_exact_residue", lambda v: int(bool(v))),
                "bicgstab-ell": ("bicgstab_ell", int),
                "jacobi-omega": ("omega", float), "sor-omega": ("omega", float),
                "residue-period": ("residue_period", int),
                "ilut-p": ("ilut_p", int), "ilut-threshold": ("ilut_threshold", float)}
        for k, v in params.items():
            k = k[len(prefix):] if prefix and k.startswith(prefix) else k
            if k == "gmres-variant":
                variants = {"CGS": 0, "CGSR": 1, "MGS": 2, "MGSR": 3, "CWY": 4}
                if v not in variants:
                    return False
                o.gmres_variant = variants[v]
            elif k == "preconditioner":
                self.setPreconditioner(v)
            elif k in keys:
                field, conv = keys[k]
                setattr(o, field, conv(v))
        self._reset()
        return True

    def _reset(self):
        if self._solver is not None:
            lib.b2s_solver_destroy(self._solver)
            self._solver = None

    def _ensure(self):
        if self._solver is None:
            if self.matrix is None:
                raise RuntimeError("No matrix was set. Call setMatrix() before solve().")
            h = C.c_void_p()
            check(lib.b2s_solver_create(self.matrix.handle, C.byref(self.opts), C.byref(h)), "b2s_solver_create")
            self._solver = h

    def solve(self, b, x, stream=None) -> bool:
        """bool solve( b, x ): x holds the initial guess and receives the solution."""
        self._ensure()
        pb, wb = _ptr(b, self.matrix.real)
        px, wx = _ptr(x, self.matrix.real)
        if wb != wx:
            raise TypeError("b and x must both be on the host or both on the device")
        st = lib.b2s_solve(self._solver, pb, px, wb, _stream_ptr(stream), C.byref(self.report))
        if st not in (OK, NOT_CONVERGED, NAN, DIVERGED, BREAKDOWN):
            raise B2SError(st, "b2s_solve")
        return st == OK

    def getIterations(self):
        return self.report.iterations

    def getResidue(self):
        return self.report.residue

    def __del__(self):
        try:
            self._reset()
        except Exception:
            pass


class CG(_LinearSolver):
    kind = _abi.CG


class BICGStab(_LinearSolver):
    kind = _abi.BICGSTAB


class GMRES(_LinearSolver):
    kind = _abi.GMRES


class TFQMR(_LinearSolver):
    """Solvers::Linear::TFQMR (TFQMR.hpp:18-114)."""
    kind = _abi.TFQMR


class _Stationary(_LinearSolver):
    def setOmega(self, omega):
        self.opts.omega = float(omega)
        self._reset()

    def getOmega(self):
        return self.opts.omega

    def setResiduePeriod(self, period):
        self.opts.residue_period = int(period)
        self._reset()

    def getResiduePeriod(self):
        return self.opts.residue_period


class Jacobi(_Stationary):
    """Solvers::Linear::Jacobi (Jacobi.hpp:67-128): weighted Jacobi sweeps."""
    kind = _abi.JACOBI


class SOR(_Stationary):
    """Solvers::Linear::SOR (SOR.hpp:66-118): the sequential forward sweep of
    TNL's Devices::Host solver, on the device as a dependency kernel."""
    kind = _abi.SOR


class BICGStabL(_LinearSolver):
    """Solvers::Linear::BICGStabL, BiCGStab(ell) (BICGStabL.hpp:42-250); ell from
    setup({"bicgstab-ell": ell}), default 1."""
    kind = _abi.BICGSTABL


# ---------------------------------------------------------------------------
# Batched solves (no TNL counterpart): many systems in one persistent launch
class BatchedCG:
    """Jacobi-PCG over a batch of independent systems (the diagonal blocks of
    one CSR matrix), 1..8 right-hand sides each, in one persistent kernel.
    B and X are torch CUDA tensors in the interleaved layout of include/b2s.h."""

    def __init__(self, offsets, columns, values, row_ptr, nrhs, tol=1e-8, preconditioner="diagonal",
                 cluster_size=0, max_iterations=None, stream=None):
        o = _abi.BatchOpts()
        lib.b2s_batch_opts_default(C.byref(o))
        o.convergence_residue = float(tol)
        o.preconditioner = 1 if preconditioner in ("diagonal", "jacobi") else 0
        o.cluster_size = int(cluster_size)
        if max_iterations is not None:
            o.max_iterations = int(max_iterations)
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int64)
        self.nrhs = np.ascontiguousarray(nrhs, np.int32)
        nsys = len(self.nrhs)
        if _is_torch(offsets):
            ptrs = [C.c_void_p(t.data_ptr()) for t in (offsets, columns, values)]
            where = DEVICE
        else:
            self._host = (np.ascontiguousarray(offsets, np.int32), np.ascontiguousarray(columns, np.int32),
                          np.ascontiguousarray(values, np.float64))
            ptrs = [C.c_void_p(a.ctypes.data) for a in self._host]
            where = HOST
        h = C.c_void_p()
        check(lib.b2s_batch_create(nsys, C.c_void_p(self.row_ptr.ctypes.data), C.c_void_p(self.nrhs.ctypes.data),
                                   *ptrs, where, C.byref(o), _stream_ptr(stream), C.byref(h)), "b2s_batch_create")
        self._h = h
        self._host = None
        n = np.diff(self.row_ptr)
        self.vec_off = np.concatenate([[0], np.cumsum(n * self.nrhs)]).astype(np.int64)
        self.rhs_off = np.concatenate([[0], np.cumsum(self.nrhs)]).astype(np.int64)
        self.report = _abi.BatchReport()

    @property
    def vector_length(self):
        return int(self.vec_off[-1])

    def solve(self, B, X, stream=None) -> bool:
        st = lib.b2s_batch_solve(self._h, C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr()), _stream_ptr(stream),
                                 C.byref(self.report))
        if st not in (OK, NOT_CONVERGED):
            raise B2SError(st, "b2s_batch_solve")
        return st == OK

    def results(self):
        m = int(self.rhs_off[-1])
        it = np.zeros(m, np.int64)
        res = np.zeros(m, np.float64)
        sts = np.zeros(m, np.int32)
        check(lib.b2s_batch_results(self._h, C.c_void_p(it.ctypes.data), C.c_void_p(res.ctypes.data),
                                    C.c_void_p(sts.ctypes.data)), "b2s_batch_results")
        return it, res, sts

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib.b2s_batch_destroy(h)
            self._h = None


# ---------------------------------------------------------------------------
# Serving (no TNL counterpart): continuous batching of solve requests
SOLVERS = {"cg": _abi.CG, "bicgstab": _abi.BICGSTAB, "gmres": _abi.GMRES, "tfqmr": _abi.TFQMR,
           "bicgstabl": _abi.BICGSTABL, "jacobi": _abi.JACOBI, "sor": _abi.SOR}


def solve_opts(solver="cg", tol=1e-10, mixed=False, preconditioner=None, gmres_variant="MGSR", restart=30,
               inner_tolerance=None, max_iterations=None):
    """b2s_solve_opts with TNL's defaults and the given overrides."""
    o = _abi.SolveOpts()
    lib.b2s_solve_opts_default(C.byref(o))
    o.solver = SOLVERS[solver]
    o.convergence_residue = float(tol)
    o.precision = _abi.PRECISION_MIXED if mixed else _abi.PRECISION_PLAIN
    o.preconditioner = 1 if preconditioner in ("diagonal", "jacobi") else 0
    o.gmres_variant = {"CGS": 0, "CGSR": 1, "MGS": 2, "MGSR": 3, "CWY": 4}[gmres_variant]
    o.gmres_restarting_min = o.gmres_restarting_max = int(restart)
    if inner_tolerance is not None:
        o.inner_tolerance = float(inner_tolerance)
    if max_iterations is not None:
        o.max_iterations = int(max_iterations)
    return o


class Server:
    """Request server of include/b2s.h: submit(csr, b, x, opts) -> ticket,
    wait(ticket) -> result dict. Host arrays are kept alive by the server
    object until their request is collected."""

    def __init__(self, memory_budget=None, max_inflight=8, mixed_min_rows=0):
        o = _abi.ServerOpts()
        lib.b2s_server_opts_default(C.byref(o))
        if memory_budget is not None:
            o.memory_budget = int(memory_budget)
        o.max_inflight = int(max_inflight)
        o.mixed_min_rows = int(mixed_min_rows)
        h = C.c_void_p()
        check(lib.b2s_server_create(C.byref(o), C.byref(h)), "b2s_server_create")
        self._h = h
        self._keep = {}

    @staticmethod
    def clock_ns():
        return lib.b2s_server_clock_ns()

    def submit(self, csr, b, x, opts, segments="CSR"):
        off, col, val = (np.ascontiguousarray(csr[0], np.int32), np.ascontiguousarray(csr[1], np.int32),
                         np.ascontiguousarray(csr[2], np.float64))
        b = np.ascontiguousarray(b, np.float64)
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
            raise TypeError("x must be a contiguous float64 numpy array (it receives the solution)")
        r = _abi.Request()
        r.format = SEGMENTS[segments]
        r.rows = len(off) - 1
        r.nnz = len(col)
        r.offsets, r.columns, r.values = off.ctypes.data, col.ctypes.data, val.ctypes.data
        r.b, r.x = b.ctypes.data, x.ctypes.data
        r.opts = opts
        t = C.c_int64()
        check(lib.b2s_server_submit(self._h, C.byref(r), C.byref(t)), "b2s_server_submit")
        self._keep[t.value] = (off, col, val, b, x)
        return t.value

    def wait(self, ticket, timeout=-1.0):
        res = _abi.RequestResult()
        st = lib.b2s_server_wait(self._h, int(ticket), float(timeout), C.byref(res))
        if st == TIMEOUT:
            return None
        check(st, "b2s_server_wait")
        self._keep.pop(ticket, None)
        rep = res.report
        return {"status": res.status, "ok": res.status == OK, "iterations": rep.iterations,
                "precision": "mixed" if res.precision == _abi.PRECISION_MIXED else "fp64",
                "refinements": rep.refinements, "residue": rep.residue, "true_residual": rep.true_residual,
                "device_ms": rep.device_ms, "t_submit_ns": res.t_submit_ns, "t_admit_ns": res.t_admit_ns,
                "t_done_ns": res.t_done_ns, "device_bytes": res.device_bytes,
                "t_built_ns": res.t_built_ns, "t_solved_ns": res.t_solved_ns,
                "error": lib.b2s_last_error().decode() if res.status != OK else ""}

    def stats(self):
        s = _abi.ServerStats()
        check(lib.b2s_server_get_stats(self._h, C.byref(s)), "b2s_server_get_stats")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.b2s_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
