"""b2s_scan_i32_noalloc: the prefix sum for callers that cannot allocate device
memory (an application whose pool allocator owns all device memory, or code
that cannot afford the synchronization of cudaFree). It must give the same
result as b2s_scan_i32, which allocates its working memory, and as numpy's
cumulative sum, on consecutive calls that reuse the library's fixed working
array — up to the largest size the array admits. This file is collected last
on purpose; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 32768 * 2048  # 67,108,864: tile totals for 32,768 tiles of 2,048 elements


def _lib():
    import b2s
    f = b2s.lib.b2s_scan_i32_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int64, C.c_void_p, C.c_int32, C.c_void_p]
    return b2s, f


def _expected(v, inclusive):
    """The scan in 64-bit sums stored as int32, as both library scans store it."""
    c = np.cumsum(v, dtype=np.int64)
    if not inclusive:
        c = np.concatenate([[0], c[:-1]])
    return c.astype(np.int32)


@pytest.mark.parametrize("inclusive", [0, 1])
def test_noalloc_scan_matches_allocating_scan_twice(cuda, inclusive):
    b2s, noalloc = _lib()
    # two calls in a row: the second must not be disturbed by what the first left in the array
    for n, seed in ((3_000_001, 1), (2049, 2)):
        v = np.random.default_rng(seed).integers(-50, 100, n).astype(np.int32)
        ref = cuda.tensor(v, device="cuda")
        got = cuda.tensor(v, device="cuda")
        b2s.check(b2s.lib.b2s_scan_i32(n, C.c_void_p(ref.data_ptr()), inclusive, None), "b2s_scan_i32")
        st = noalloc(n, got.data_ptr(), inclusive, None)
        assert st == b2s.OK, b2s.lib.b2s_last_error()
        cuda.cuda.synchronize()  # the call only queues its kernels
        assert cuda.equal(got, ref)
        assert np.array_equal(got.cpu().numpy(), _expected(v, inclusive))


def test_noalloc_scan_at_the_size_limit(cuda):
    b2s, noalloc = _lib()
    # the largest admitted size, then a small call that reuses the array after it
    for n, seed, inclusive in ((MAX_N, 3, 0), (MAX_N, 4, 1), (5, 5, 0)):
        v = np.random.default_rng(seed).integers(-3, 4, n).astype(np.int32)
        got = cuda.tensor(v, device="cuda")
        assert noalloc(n, got.data_ptr(), inclusive, None) == b2s.OK, b2s.lib.b2s_last_error()
        cuda.cuda.synchronize()
        assert np.array_equal(got.cpu().numpy(), _expected(v, inclusive))
        del got


def test_noalloc_scan_rejects_oversize(cuda):
    b2s, noalloc = _lib()
    t = cuda.zeros(16, dtype=cuda.int32, device="cuda")
    assert noalloc(MAX_N + 1, t.data_ptr(), 0, None) == b2s.INVALID_ARG
    assert b"exceeds" in b2s.lib.b2s_last_error()
    assert noalloc(16, t.data_ptr(), 0, None) == b2s.OK
