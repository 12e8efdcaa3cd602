"""Algorithms primitives on the GPU (reduce / scan / vector update) against
numpy, mirroring TNL's reduceTest / scanTest (src/UnitTests/Algorithms)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 31, 257, 100_003, 5_000_000])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_dot_and_norm(b2s_lib, cuda, n, dtype):
    rng = np.random.default_rng(n)
    a = rng.uniform(-1, 1, n).astype(dtype)
    b = rng.uniform(-1, 1, n).astype(dtype)
    ta, tb = cuda.tensor(a, device="cuda"), cuda.tensor(b, device="cuda")
    res = cuda.zeros(2, dtype=cuda.float64, device="cuda")
    b2s_lib.dot(ta, tb, res[0:1])
    b2s_lib.norm2(ta, res[1:2])
    d, nr = res.cpu().numpy()
    ref_d = float(np.dot(a.astype(np.float64), b.astype(np.float64)))
    ref_n = float(np.sqrt(np.dot(a.astype(np.float64), a.astype(np.float64))))
    assert abs(d - ref_d) <= 1e-12 * max(1.0, np.abs(a.astype(np.float64) * b).sum())
    assert abs(nr - ref_n) <= 1e-12 * max(1.0, ref_n)
    # deterministic: the same inputs give the same bits
    res2 = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    b2s_lib.dot(ta, tb, res2)
    assert float(res2[0]) == d


@pytest.mark.parametrize("n", [1, 1000, 3_000_001])
def test_axpby(b2s_lib, cuda, n):
    rng = np.random.default_rng(1)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    tx, ty = cuda.tensor(x, device="cuda"), cuda.tensor(y, device="cuda")
    b2s_lib.axpby(2.5, tx, -0.5, ty)
    assert np.allclose(ty.cpu().numpy(), 2.5 * x + -0.5 * y, rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 1_000_000, 9_000_001])
@pytest.mark.parametrize("inclusive", [False, True])
def test_scan(b2s_lib, cuda, n, inclusive):
    rng = np.random.default_rng(n)
    v = rng.integers(0, 100, n).astype(np.int32)
    t = cuda.tensor(v, device="cuda")
    b2s_lib.scan_i32(t, inclusive)
    c = np.cumsum(v.astype(np.int64))
    ref = c if inclusive else np.concatenate([[0], c[:-1]])
    assert np.array_equal(t.cpu().numpy().astype(np.int64), ref)
