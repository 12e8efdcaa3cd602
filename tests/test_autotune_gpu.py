"""The SpMV layout autotuner (b2s_autotune_spmv): every candidate it times is
a valid layout, the reported best is the fastest of them, the CSR entries name
the kernel that was built, and the chosen configuration rebuilt through
b2s_matrix_create gives TNL's product (oracle, 1e-12 relative in FP64); cold
(L2 evicted, the default) and warm timings both run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["laplace", "irregular"])
def test_autotune_picks_the_fastest_valid_layout(b2s_lib, cuda, oracle, kind):
    from b2s import workloads as W
    csr = W.laplace3d(40) if kind == "laplace" else W.irregular(60000, seed=5, hi=900)
    A = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    best, table = b2s_lib.autotune(A, reps=5)
    timed = [e for e in table if not e["skipped"]]
    assert len(timed) >= 5
    assert best["spmv_us"] == pytest.approx(min(e["spmv_us"] for e in timed))
    names = {e["segments"] for e in table}
    assert names == {"CSR", "Ellpack", "SlicedEllpack", "ChunkedEllpack", "BiEllpack", "Multidiagonal"}
    assert {e["slice_size"] for e in table if e["segments"] == "SlicedEllpack"} == {8, 16, 32, 64}
    adaptive = [e for e in table if e["csr_kernel"] == "CSRAdaptive"]
    # the 32-row group kernel is a candidate where every group fits (the stencil), beside the
    # windows; the entries name the kernel that was built (the irregular rows get windows)
    assert [e["csr_row_groups"] for e in adaptive] == ([True, False] if kind == "laplace" else [False])
    if kind == "irregular":
        # max row 900 against a mean of ~15: Ellpack padding is far above the limit
        assert next(e for e in table if e["segments"] == "Ellpack")["skipped"]
    kw = {k: best[k] for k in ("segments", "csr_kernel", "threads_per_row", "slice_size", "csr_row_groups")}
    M = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3], **kw)
    x = W.uniform(csr[3], 3)
    y = np.zeros(len(csr[0]) - 1)
    M.vectorProduct(x, y)
    ref = oracle.spmv("csr", "col", csr, x)
    assert np.max(np.abs(y - ref)) / np.max(np.abs(ref)) <= 1e-12


def test_autotune_warm_l2_option(b2s_lib, cuda):
    from b2s import workloads as W
    csr = W.laplace3d(24)
    A = b2s_lib.SparseMatrix.from_csr(*csr[:3], csr[3])
    cold, _ = b2s_lib.autotune(A, reps=3)
    warm, _ = b2s_lib.autotune(A, reps=3, warm_l2=True)
    assert cold["spmv_us"] > 0 and warm["spmv_us"] > 0
